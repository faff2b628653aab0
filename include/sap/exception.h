/* sap::system_error for the C ABI of libsap_b200 (include/sap_b200.h):
 * the reference's exception type (sap/exception.h:13-45), with the same
 * Reason values, raised from the library's status codes; library failures
 * that have no reference counterpart (CUDA errors, invalid arguments,
 * unsupported options, a bounded device wait that ran out) raise
 * sap::library_error. */
#ifndef SAP_B200_FACADE_EXCEPTION_H
#define SAP_B200_FACADE_EXCEPTION_H

#include <stdexcept>
#include <string>

#include "../sap_b200.h"

namespace sap {

class system_error : public std::runtime_error {
 public:
  enum Reason {
    Zero_pivoting = SAP_ZERO_PIVOTING,
    Negative_DB_weight = SAP_NEGATIVE_DB_WEIGHT,
    Illegal_update = SAP_ILLEGAL_UPDATE,
    Illegal_solve = SAP_ILLEGAL_SOLVE,
    Matrix_singular = SAP_MATRIX_SINGULAR
  };
  system_error(Reason reason, const std::string& what_arg) : std::runtime_error(what_arg), m_reason(reason) {}
  Reason reason() const { return m_reason; }

 private:
  Reason m_reason;
};

class library_error : public std::runtime_error {
 public:
  library_error(int code, const std::string& what_arg) : std::runtime_error(what_arg), m_code(code) {}
  int code() const { return m_code; }

 private:
  int m_code;
};

namespace detail {
// Turns a status of the C ABI into the exception the reference would raise.
inline void check(int code) {
  if (code == SAP_OK) return;
  const char* m = sap_last_error();
  const std::string msg = m ? m : "";
  if (code <= SAP_ZERO_PIVOTING && code >= SAP_MATRIX_SINGULAR)
    throw system_error(static_cast<system_error::Reason>(code), msg);
  throw library_error(code, msg);
}
}  // namespace detail

}  // namespace sap

#endif
