/* Helpers of the C++ facade: raw pointers and memory spaces of the caller's
 * containers.  A container is anything with data() and size() whose data()
 * is a raw pointer or a fancy pointer with get() (thrust::device_ptr and
 * the like); its memory space is looked up with cudaPointerGetAttributes. */
#ifndef SAP_B200_FACADE_DETAIL_H
#define SAP_B200_FACADE_DETAIL_H

#include <cuda_runtime.h>

#include "../sap_b200.h"

namespace sap {
namespace detail {

template <typename T>
T* raw(T* p) { return p; }
template <typename P>
auto raw(P p) -> decltype(p.get()) { return p.get(); }

template <typename V>
auto data_of(V& v) -> decltype(raw(v.data())) { return raw(v.data()); }
template <typename V>
auto data_of(const V& v) -> decltype(raw(v.data())) { return raw(v.data()); }

// SAP_DEVICE for device or managed memory, SAP_HOST otherwise
inline int memspace(const void* p) {
  cudaPointerAttributes a{};
  if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return SAP_HOST;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ? SAP_DEVICE : SAP_HOST;
}

template <typename T>
struct prec_code;
template <>
struct prec_code<float> { static constexpr int value = SAP_PREC_FLOAT; };
template <>
struct prec_code<double> { static constexpr int value = SAP_PREC_DOUBLE; };

}  // namespace detail
}  // namespace sap

#endif
