/* The SpMV functors of the reference (sap/spmv.h:27-129) over the C ABI:
 * SpmvCusp<Matrix> for a CSR matrix (FP64 values, int32 indices; the
 * members num_rows, num_entries, row_offsets, column_indices, values of a
 * CUSP-style csr_matrix, on the host or the device) and MVBanded<Matrix>
 * for a sap::BandedMatrix.  The reference functors keep a reference to the
 * caller's matrix; SpmvCusp here keeps the library's device copy of it,
 * made at construction.  operator()(v, Av) runs on the device. */
#ifndef SAP_B200_FACADE_SPMV_H
#define SAP_B200_FACADE_SPMV_H

#include "banded_matrix.h"
#include "detail.h"
#include "exception.h"

namespace sap {

// A CSR matrix (CUSP member names) as the library's device CSR.
template <typename Matrix>
sap_csr* make_csr(const Matrix& A) {
  const int* rp = detail::data_of(A.row_offsets);
  const int* ci = detail::data_of(A.column_indices);
  const double* v = detail::data_of(A.values);
  sap_csr* h = nullptr;
  detail::check(sap_csr_create((int)A.num_rows, (int)A.num_entries, rp, ci, v, detail::memspace(v), &h));
  return h;
}

template <typename Matrix>
class SpmvCusp {
 public:
  explicit SpmvCusp(const Matrix& A) : m_A(make_csr(A)) { detail::check(sap_spmv_csr_create(m_A, &m_h)); }
  ~SpmvCusp() {
    if (m_h) sap_spmv_destroy(m_h);
    if (m_A) sap_csr_destroy(m_A);
  }
  SpmvCusp(const SpmvCusp&) = delete;
  SpmvCusp& operator=(const SpmvCusp&) = delete;

  template <typename Array>
  void operator()(const Array& v, Array& Av) {
    detail::check(sap_spmv_apply(m_h, detail::data_of(v), detail::data_of(Av)));
  }
  // timing counters of the reference's functor (stubs there too, spmv.h:96-108)
  double getTime() const { return 0.0; }
  double getCount() const { return 0.0; }
  double getGFlops() const { return 0.0; }
  sap_spmv* handle() const { return m_h; }

 private:
  sap_csr* m_A = nullptr;
  sap_spmv* m_h = nullptr;
};

template <typename Matrix>
class MVBanded {
 public:
  explicit MVBanded(const Matrix& A) { detail::check(sap_spmv_banded_create(A.handle(), &m_h)); }
  ~MVBanded() {
    if (m_h) sap_spmv_destroy(m_h);
  }
  MVBanded(const MVBanded&) = delete;
  MVBanded& operator=(const MVBanded&) = delete;

  template <typename Array>
  void operator()(const Array& v, Array& Av) {
    detail::check(sap_spmv_apply(m_h, detail::data_of(v), detail::data_of(Av)));
  }
  double getTime() const { return 0.0; }
  double getCount() const { return 0.0; }
  double getGFlops() const { return 0.0; }
  sap_spmv* handle() const { return m_h; }

 private:
  sap_spmv* m_h = nullptr;
};

}  // namespace sap

#endif
