/* sap::Options, sap::Stats and sap::Solver<Array, PrecValueType> of the
 * reference (sap/solver.h:52-225) over the C ABI of libsap_b200: the same
 * field names and defaults, the same member functions (setup, update,
 * solve, getStats, getMonitorCode, getMonitorMessage), failures raised as
 * sap::system_error with the reference's Reason values.  Array is the
 * caller's FP64 vector type (data() and size(); host or device memory);
 * PrecValueType float or double selects the preconditioner's value type as
 * in the reference.  solve() takes the facade's SpmvCusp or MVBanded.
 *
 *   sap::Options opts;  opts.relTol = 1e-10;
 *   sap::Solver<Vector, float> solver(numPartitions, opts);
 *   sap::SpmvCusp<Matrix> spmv(A);
 *   solver.setup(A);
 *   bool ok = solver.solve(spmv, b, x);
 */
#ifndef SAP_B200_FACADE_SOLVER_H
#define SAP_B200_FACADE_SOLVER_H

#include <string>
#include <type_traits>

#include "banded_matrix.h"
#include "common.h"
#include "detail.h"
#include "exception.h"
#include "spmv.h"

namespace sap {

// sap::Options (sap/solver.h:52-81, defaults 233-256)
struct Options {
  KrylovSolverType solverType;
  int maxNumIterations;
  double relTol;
  double absTol;
  bool testDB;
  bool isSPD;
  bool saveMem;
  bool performReorder;
  bool performDB;
  bool dbFirstStageOnly;
  bool applyScaling;
  int maxBandwidth;
  int gpuCount;
  double dropOffFraction;
  FactorizationMethod factMethod;
  PreconditionerType precondType;
  bool safeFactorization;
  bool variableBandwidth;
  bool trackReordering;
  bool useBCR;
  int ilu_level;
  int refinementSweeps;  // extension: FP64 refinement sweeps (0: the reference's single solve)

  Options() {
    sap_options o;
    detail::check(sap_options_default(&o));
    solverType = static_cast<KrylovSolverType>(o.solverType);
    maxNumIterations = o.maxNumIterations;
    relTol = o.relTol;
    absTol = o.absTol;
    testDB = o.testDB != 0;
    isSPD = o.isSPD != 0;
    saveMem = o.saveMem != 0;
    performReorder = o.performReorder != 0;
    performDB = o.performDB != 0;
    dbFirstStageOnly = o.dbFirstStageOnly != 0;
    applyScaling = o.applyScaling != 0;
    maxBandwidth = o.maxBandwidth;
    gpuCount = o.gpuCount;
    dropOffFraction = o.dropOffFraction;
    factMethod = static_cast<FactorizationMethod>(o.factMethod);
    precondType = static_cast<PreconditionerType>(o.precondType);
    safeFactorization = o.safeFactorization != 0;
    variableBandwidth = o.variableBandwidth != 0;
    trackReordering = o.trackReordering != 0;
    useBCR = o.useBCR != 0;
    ilu_level = o.ilu_level;
    refinementSweeps = o.refinementSweeps;
  }
  sap_options c() const {
    sap_options o;
    o.solverType = solverType;
    o.maxNumIterations = maxNumIterations;
    o.relTol = relTol;
    o.absTol = absTol;
    o.testDB = testDB;
    o.isSPD = isSPD;
    o.saveMem = saveMem;
    o.performReorder = performReorder;
    o.performDB = performDB;
    o.dbFirstStageOnly = dbFirstStageOnly;
    o.applyScaling = applyScaling;
    o.maxBandwidth = maxBandwidth;
    o.gpuCount = gpuCount;
    o.dropOffFraction = dropOffFraction;
    o.factMethod = factMethod;
    o.precondType = precondType;
    o.safeFactorization = safeFactorization;
    o.variableBandwidth = variableBandwidth;
    o.trackReordering = trackReordering;
    o.useBCR = useBCR;
    o.ilu_level = ilu_level;
    o.refinementSweeps = refinementSweeps;
    return o;
  }
};

// sap::Stats (sap/solver.h:89-140): the same fields, times in milliseconds
typedef sap_stats Stats;

template <typename Array, typename PrecValueType = double>
class Solver {
 public:
  Solver(int numPartitions, const Options& opts) : m_opts(opts) {
    const sap_options o = opts.c();
    detail::check(sap_solver_create(numPartitions, &o, detail::prec_code<PrecValueType>::value, &m_h));
  }
  virtual ~Solver() {
    if (m_h) sap_solver_destroy(m_h);
    if (m_A) sap_csr_destroy(m_A);
  }
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;

  // setup(A) for a sap::BandedMatrix
  template <typename Array2>
  bool setup(const BandedMatrix<Array2>& A) {
    detail::check(sap_solver_setup_banded(m_h, A.handle()));
    return true;
  }
  // setup(A) for a CSR matrix (CUSP member names, FP64 values)
  template <typename Matrix>
  bool setup(const Matrix& A) {
    if (m_A) sap_csr_destroy(m_A);
    m_A = nullptr;
    m_A = make_csr(A);
    detail::check(sap_solver_setup_csr(m_h, m_A));
    return true;
  }
  // update(entries): false when the number of entries differs from the setup matrix's
  template <typename Array1>
  bool update(const Array1& entries) {
    const double* e = detail::data_of(entries);
    int accepted = 1;
    detail::check(sap_solver_update(m_h, e, (int64_t)entries.size(), detail::memspace(e), &accepted));
    return accepted != 0;
  }
  // solve(spmv, b, x): x holds the initial guess and receives the solution
  template <typename SpmvOperator>
  bool solve(SpmvOperator& spmv, const Array& b, Array& x) {
    const double* pb = detail::data_of(b);
    double* px = detail::data_of(x);
    int conv = 0;
    detail::check(sap_solver_solve(m_h, spmv.handle(), pb, px, detail::memspace(px), &conv));
    return conv != 0;
  }
  const Stats& getStats() const {
    detail::check(sap_solver_get_stats(m_h, &m_stats));
    return m_stats;
  }
  int getMonitorCode() const {
    int code = 0;
    detail::check(sap_solver_get_monitor(m_h, &code, nullptr));
    return code;
  }
  const std::string& getMonitorMessage() const {
    const char* m = nullptr;
    detail::check(sap_solver_get_monitor(m_h, nullptr, &m));
    m_msg = m ? m : "";
    return m_msg;
  }

 private:
  Options m_opts;
  sap_solver* m_h = nullptr;
  sap_csr* m_A = nullptr;
  mutable Stats m_stats{};
  mutable std::string m_msg;
};

}  // namespace sap

#endif
