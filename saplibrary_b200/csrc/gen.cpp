// Synthetic banded matrices (the reference's BandedMatrix generator,
// sap/banded_matrix.h:59-95, plus seeded counter-based variants).
#include <cmath>
#include <cstdint>
#include <cstdlib>

#include "reorder.h"

namespace sapb {

static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
// uniform in [0,1) from 53 random bits
static inline double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

void generate_band(int n, int k, double d, int dist, uint64_t seed, double* A) {
  const long long SW = 2LL * k + 1;
  if (dist == 0) {
    // The reference generator: rand() in [-10, 10] for every in-range
    // position of the row (the diagonal's draw is discarded), the diagonal
    // set to d * sum |off-diagonals| (sap/banded_matrix.h:73-92).
    srand((unsigned)seed);
    for (int ir = 0; ir < n; ir++) {
      int left = ir - k < 0 ? 0 : ir - k;
      int right = ir + k > n - 1 ? n - 1 : ir + k;
      double row_sum = 0;
      double* row = A + (long long)ir * SW + k - ir;
      for (int ic = left; ic <= right; ic++) {
        double val = -10.0 + 20.0 * rand() / RAND_MAX;
        if (ir != ic) {
          row_sum += std::fabs(val);
          row[ic] = val;
        }
      }
      row[ir] = d * row_sum;
    }
    return;
  }
  const uint64_t s0 = splitmix64(seed ^ 0x5A5A5A5A12345678ULL);
#pragma omp parallel for schedule(static)
  for (int ir = 0; ir < n; ir++) {
    int left = ir - k < 0 ? 0 : ir - k;
    int right = ir + k > n - 1 ? n - 1 : ir + k;
    double row_sum = 0;
    double* row = A + (long long)ir * SW + k - ir;
    for (int ic = left; ic <= right; ic++) {
      if (ic == ir) continue;
      uint64_t h = splitmix64(s0 ^ splitmix64(((uint64_t)ir << 32) | (uint32_t)ic));
      double val;
      if (dist == 1) {
        val = -1.0 + 2.0 * u01(h);
      } else {
        // Box-Muller on two decorrelated draws
        double u1 = u01(h), u2 = u01(splitmix64(h));
        if (u1 < 1e-300) u1 = 1e-300;
        val = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
      }
      row[ic] = val;
      row_sum += std::fabs(val);
    }
    row[ir] = d * row_sum;
  }
}

}  // namespace sapb
