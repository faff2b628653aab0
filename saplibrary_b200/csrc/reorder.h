// Host-side pieces shared by the solver: the sparse reordering state and
// the synthetic banded-matrix generator.
#pragma once

#include <cstdint>
#include <vector>

namespace sapb {

class PrecBase;
struct Csr;

// Permutations and scalings of the reordered sparse path
// (Precond::m_optPerm / m_optReordering / m_dbRowScale / m_dbColScale,
// sap/precond.h:235-245).
struct Reorder {
  std::vector<int> perm_in;      // row i of A goes to row perm_in[i] of the band
  std::vector<int> perm_out;     // band row j goes to solution row perm_out[j]
  std::vector<double> scale_in;  // DB row scale (per original row)
  std::vector<double> scale_out; // DB column scale (per original column)
};

void reorder_setup(PrecBase& pc, const Csr& A);
void reorder_apply_in(PrecBase& pc, const double* v, double* out);
void reorder_apply_out(PrecBase& pc, const double* in, double* z);

// BandedMatrix(n, k, d) generator (sap/banded_matrix.h:59-95), row-major.
void generate_band(int n, int k, double d, int dist, uint64_t seed, double* out);

}  // namespace sapb
