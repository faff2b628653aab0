/* sap::BandedMatrix<Array> (sap/banded_matrix.h:25-95 of the reference):
 * the synthetic banded matrix of order n, half-bandwidth k and diagonal
 * dominance d.  As in the reference, every in-range position of row i
 * draws -10 + 20 rand() / RAND_MAX from the caller's rand() stream (the
 * diagonal's draw is discarded), off-diagonals keep their draws and the
 * diagonal is d times the row's sum of |off-diagonals|; the row-major band
 * (2k+1 values per row) is then uploaded to the device through
 * sap_banded_create. */
#ifndef SAP_B200_FACADE_BANDED_MATRIX_H
#define SAP_B200_FACADE_BANDED_MATRIX_H

#include <cmath>
#include <cstdlib>
#include <vector>

#include "exception.h"

namespace sap {

template <typename Array>
class BandedMatrix {
 public:
  typedef typename Array::value_type value_type;
  typedef int index_type;

  BandedMatrix(int n, int k, double d) : m_n(n), m_k(k), num_rows(n), num_cols(n), m_d(d) {
    num_entries = (size_t)n * (2 * k + 1) - (size_t)k * (k + 1);
    std::vector<double> A((size_t)n * (2 * k + 1), 0.0);
    size_t middle = (size_t)k;
    for (int ir = 0; ir < n; ir++) {
      const int left = ir - k < 0 ? 0 : ir - k, right = ir + k > n - 1 ? n - 1 : ir + k;
      value_type row_sum = 0;
      for (int ic = left; ic <= right; ic++) {
        const value_type val = -10.0 + 20.0 * rand() / RAND_MAX;
        if (ir != ic) {
          row_sum += std::abs(val);
          A[middle + ic - ir] = val;
        }
      }
      A[middle] = d * row_sum;
      middle += 2 * k + 1;
    }
    detail::check(sap_banded_create(n, k, A.data(), SAP_HOST, &m_h));
  }
  ~BandedMatrix() {
    if (m_h) sap_banded_destroy(m_h);
  }
  BandedMatrix(const BandedMatrix&) = delete;
  BandedMatrix& operator=(const BandedMatrix&) = delete;

  // the row-major band (2k+1 values per row), copied to the host
  std::vector<double> getBandedMatrix() const {
    std::vector<double> out((size_t)m_n * (2 * m_k + 1));
    detail::check(sap_banded_copy_out(m_h, out.data(), SAP_HOST));
    return out;
  }
  const sap_banded* handle() const { return m_h; }

  int m_n, m_k;
  int num_rows, num_cols;
  size_t num_entries;

 private:
  double m_d;
  sap_banded* m_h = nullptr;
};

}  // namespace sap

#endif
