// ORACLE — test infrastructure only.  A minimal stand-in for the parts of
// CUSP (github.com/cusplibrary, absent from this image) that the reference's
// sap/graph.h uses, so that graph.h itself can be compiled and run as the
// parity reference of the reordering pipeline.  It restates CUSP's
// documented container semantics on top of Thrust:
//   cusp::array1d<T, host_memory | device_memory>  a Thrust host / device vector
//   cusp::csr_matrix / cusp::coo_matrix            num_rows, num_cols, num_entries and the index / value arrays
//   cusp::blas::fill                               fill an array with a value
//   cusp::offsets_to_indices / indices_to_offsets  CSR row offsets <-> sorted row indices
// and the Thrust headers that CUSP's headers bring in for graph.h.
#pragma once

#include <thrust/binary_search.h>
#include <thrust/copy.h>
#include <thrust/count.h>
#include <thrust/device_vector.h>
#include <thrust/extrema.h>
#include <thrust/fill.h>
#include <thrust/functional.h>
#include <thrust/gather.h>
#include <thrust/host_vector.h>
#include <thrust/inner_product.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/discard_iterator.h>
#include <thrust/iterator/transform_iterator.h>
#include <thrust/logical.h>
#include <thrust/reduce.h>
#include <thrust/scan.h>
#include <thrust/scatter.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/transform_reduce.h>

#include <cstddef>


namespace cusp {

struct host_memory {};
struct device_memory {};

namespace shim_detail {
template <typename T, typename Mem>
struct vec;
template <typename T>
struct vec<T, host_memory> {
  typedef thrust::host_vector<T> type;
};
template <typename T>
struct vec<T, device_memory> {
  typedef thrust::device_vector<T> type;
};
}  // namespace shim_detail

template <typename T, typename Mem>
class array1d : public shim_detail::vec<T, Mem>::type {
  typedef typename shim_detail::vec<T, Mem>::type Base;

 public:
  typedef Mem memory_space;
  array1d() {}
  explicit array1d(std::size_t n) : Base(n) {}
  array1d(std::size_t n, const T& value) : Base(n, value) {}
  array1d(const array1d& o) : Base(o) {}
  template <typename T2, typename M2>
  array1d(const array1d<T2, M2>& o) : Base(o.begin(), o.end()) {}
  template <typename It>
  array1d(It first, It last) : Base(first, last) {}
  array1d& operator=(const array1d& o) {
    Base::operator=(o);
    return *this;
  }
  template <typename T2, typename M2>
  array1d& operator=(const array1d<T2, M2>& o) {
    Base::assign(o.begin(), o.end());
    return *this;
  }
};

template <typename I, typename V, typename Mem>
struct coo_matrix {
  typedef I index_type;
  typedef V value_type;
  typedef Mem memory_space;
  std::size_t num_rows = 0, num_cols = 0, num_entries = 0;
  array1d<I, Mem> row_indices, column_indices;
  array1d<V, Mem> values;
  coo_matrix() {}
  coo_matrix(std::size_t r, std::size_t c, std::size_t nnz)
      : num_rows(r), num_cols(c), num_entries(nnz), row_indices(nnz), column_indices(nnz), values(nnz) {}
  template <typename I2, typename V2, typename M2>
  coo_matrix(const coo_matrix<I2, V2, M2>& o)
      : num_rows(o.num_rows), num_cols(o.num_cols), num_entries(o.num_entries), row_indices(o.row_indices),
        column_indices(o.column_indices), values(o.values) {}
  void resize(std::size_t r, std::size_t c, std::size_t nnz) {
    num_rows = r;
    num_cols = c;
    num_entries = nnz;
    row_indices.resize(nnz);
    column_indices.resize(nnz);
    values.resize(nnz);
  }
};

template <typename I, typename V, typename Mem>
struct csr_matrix {
  typedef I index_type;
  typedef V value_type;
  typedef Mem memory_space;
  std::size_t num_rows = 0, num_cols = 0, num_entries = 0;
  array1d<I, Mem> row_offsets, column_indices;
  array1d<V, Mem> values;
  csr_matrix() : row_offsets(1, I(0)) {}
  csr_matrix(std::size_t r, std::size_t c, std::size_t nnz)
      : num_rows(r), num_cols(c), num_entries(nnz), row_offsets(r + 1), column_indices(nnz), values(nnz) {}
  template <typename I2, typename V2, typename M2>
  csr_matrix(const csr_matrix<I2, V2, M2>& o)
      : num_rows(o.num_rows), num_cols(o.num_cols), num_entries(o.num_entries), row_offsets(o.row_offsets),
        column_indices(o.column_indices), values(o.values) {}
  template <typename I2, typename V2, typename M2>
  csr_matrix& operator=(const csr_matrix<I2, V2, M2>& o) {
    num_rows = o.num_rows;
    num_cols = o.num_cols;
    num_entries = o.num_entries;
    row_offsets = o.row_offsets;
    column_indices = o.column_indices;
    values = o.values;
    return *this;
  }
  // COO -> CSR: a stable counting sort of the entries by row (CUSP's
  // conversion; for entries already sorted by row it is a plain copy)
  template <typename I2, typename V2, typename M2>
  csr_matrix& operator=(const coo_matrix<I2, V2, M2>& o) {
    thrust::host_vector<I2> ri(o.row_indices.begin(), o.row_indices.end());
    thrust::host_vector<I2> cj(o.column_indices.begin(), o.column_indices.end());
    thrust::host_vector<V2> va(o.values.begin(), o.values.end());
    const std::size_t nnz = o.num_entries;
    thrust::host_vector<I> off(o.num_rows + 1, I(0));
    for (std::size_t e = 0; e < nnz; e++) off[ri[e] + 1]++;
    for (std::size_t r = 0; r < o.num_rows; r++) off[r + 1] += off[r];
    thrust::host_vector<I> cols(nnz);
    thrust::host_vector<V> vals(nnz);
    thrust::host_vector<I> next(off.begin(), off.end() - 1);
    for (std::size_t e = 0; e < nnz; e++) {
      const I d = next[ri[e]]++;
      cols[d] = (I)cj[e];
      vals[d] = (V)va[e];
    }
    resize(o.num_rows, o.num_cols, nnz);
    thrust::copy(off.begin(), off.end(), row_offsets.begin());
    thrust::copy(cols.begin(), cols.end(), column_indices.begin());
    thrust::copy(vals.begin(), vals.end(), values.begin());
    return *this;
  }
  void resize(std::size_t r, std::size_t c, std::size_t nnz) {
    num_rows = r;
    num_cols = c;
    num_entries = nnz;
    row_offsets.resize(r + 1);
    column_indices.resize(nnz);
    values.resize(nnz);
  }
};

// indices[k] = the row whose offset range [offsets[i], offsets[i+1]) holds k
template <typename OffsetArray, typename IndexArray>
void offsets_to_indices(const OffsetArray& offsets, IndexArray& indices) {
  typedef typename IndexArray::value_type I;
  thrust::upper_bound(offsets.begin() + 1, offsets.end(), thrust::counting_iterator<I>(0),
                      thrust::counting_iterator<I>((I)indices.size()), indices.begin());
}

// offsets[i] = the first position of row i in the sorted row indices
template <typename IndexArray, typename OffsetArray>
void indices_to_offsets(const IndexArray& indices, OffsetArray& offsets) {
  typedef typename OffsetArray::value_type I;
  thrust::lower_bound(indices.begin(), indices.end(), thrust::counting_iterator<I>(0),
                      thrust::counting_iterator<I>((I)offsets.size()), offsets.begin());
}

namespace blas {
template <typename Array, typename Value>
void fill(Array& a, const Value& v) {
  thrust::fill(a.begin(), a.end(), (typename Array::value_type)v);
}
}  // namespace blas

}  // namespace cusp
