// A C++ caller written against the sap:: facade (include/sap/*.h) the way
// reference code is written against sap/solver.h and sap/spmv.h: Options,
// Solver<Array, PrecValueType>, SpmvCusp over a CSR matrix with CUSP's
// member names, MVBanded over a BandedMatrix, system_error.  Linked against
// libsap_b200.so.  Case 1 is the configuration of the reference's unit test
// (examples/unit_test/driver_unit_test.cu:49-94: N = 10,000, K = 20, 10
// partitions, dominance 1, RAND(-10, 10) values from glibc rand() in its
// default state, x(t) = 400 t (1 - t), LU_UL, no reordering, relTol 1e-13),
// with an FP64 preconditioner (in the reference's FP32 mixed mode
// BiCGStab(2) stagnates near FP32 accuracy before 1e-13).  Case 2 is a
// BandedMatrix of order 20,000, K 16, dominance 1 (FP32 preconditioner,
// relTol 1e-6) solved through MVBanded.  Case 3 checks that an illegal call
// order raises sap::system_error.  Prints one JSON line; exit 0 when every
// check holds.
#include <sap/solver.h>

#include <thrust/device_vector.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

// a CSR matrix with the member names of cusp::csr_matrix (host storage)
struct HostCsr {
  int num_rows = 0, num_cols = 0, num_entries = 0;
  std::vector<int> row_offsets, column_indices;
  std::vector<double> values;
};

static HostCsr unit_test_matrix(int N, int k, double d) {
  HostCsr A;
  A.num_rows = A.num_cols = N;
  A.row_offsets.push_back(0);
  for (int ir = 0; ir < N; ir++) {
    const int left = ir - k < 0 ? 0 : ir - k, right = ir + k > N - 1 ? N - 1 : ir + k;
    double row_sum = 0;
    size_t diag = 0;
    for (int ic = left; ic <= right; ic++) {
      const double val = -10.0 + 20.0 * (float)rand() / (float)RAND_MAX;
      if (ic == ir) diag = A.values.size();
      else row_sum += std::fabs(val);
      A.column_indices.push_back(ic);
      A.values.push_back(val);
    }
    A.values[diag] = d * row_sum;
    A.row_offsets.push_back((int)A.values.size());
  }
  A.num_entries = (int)A.values.size();
  return A;
}

int main() {
  typedef thrust::device_vector<double> Vector;
  bool pass = true;
  // ---- case 1: the unit-test configuration through SpmvCusp ----
  const int N = 10000;
  HostCsr A = unit_test_matrix(N, 20, 1.0);
  std::vector<double> xt(N), bh(N, 0.0);
  for (int i = 0; i < N; i++) {
    const double t = (double)i / (N - 1);
    xt[i] = 400.0 * t * (1.0 - t);
  }
  for (int i = 0; i < N; i++)
    for (int e = A.row_offsets[i]; e < A.row_offsets[i + 1]; e++) bh[i] += A.values[e] * xt[A.column_indices[e]];
  Vector b(bh.begin(), bh.end()), x(N, 0.0);
  sap::Options opts;
  opts.trackReordering = false;
  opts.variableBandwidth = false;
  opts.factMethod = sap::LU_UL;
  opts.performReorder = false;
  opts.applyScaling = false;
  opts.relTol = 1e-13;
  sap::Solver<Vector, double> solver(10, opts);
  sap::SpmvCusp<HostCsr> spmv(A);
  solver.setup(A);
  const bool ok1 = solver.solve(spmv, b, x);
  const int code1 = solver.getMonitorCode();
  const std::string msg1 = solver.getMonitorMessage();
  const double rel1 = solver.getStats().relResidualNorm;
  std::vector<double> xh(N);
  thrust::copy(x.begin(), x.end(), xh.begin());
  double err = 0, nrm = 0;
  for (int i = 0; i < N; i++) {
    err += (xh[i] - xt[i]) * (xh[i] - xt[i]);
    nrm += xt[i] * xt[i];
  }
  const double rel_err = std::sqrt(err / nrm);
  pass = pass && ok1 && code1 == 1 && msg1 == "Converged" && rel1 <= 1e-13 && rel_err <= 1e-9;

  // ---- case 2: BandedMatrix + MVBanded, FP32 preconditioner ----
  sap::BandedMatrix<Vector> B(20000, 16, 1.0);
  sap::MVBanded<sap::BandedMatrix<Vector> > mv(B);
  Vector ones(20000, 1.0), rhs(20000, 0.0), y(20000, 0.0);
  mv(ones, rhs);
  sap::Options o2;
  o2.performReorder = false;
  o2.variableBandwidth = false;
  o2.factMethod = sap::LU_UL;
  o2.applyScaling = false;
  sap::Solver<Vector, float> s2(4, o2);
  s2.setup(B);
  const bool ok2 = s2.solve(mv, rhs, y);
  const double rel2 = s2.getStats().relResidualNorm;
  pass = pass && ok2 && s2.getMonitorCode() == 1 && rel2 <= 1e-6;

  // ---- case 3: solve before setup raises sap::system_error ----
  int reason = 0;
  try {
    sap::Solver<Vector, double> s3(2, opts);
    s3.solve(spmv, b, x);
  } catch (const sap::system_error& e) {
    reason = (int)e.reason();
  }
  pass = pass && reason == sap::system_error::Illegal_solve;

  std::printf("{\"unit_test_converged\": %s, \"code\": %d, \"message\": \"%s\", \"rel_residual\": %.3e, "
              "\"rel_error\": %.3e, \"iterations\": %.2f, \"banded_converged\": %s, \"banded_rel_residual\": %.3e, "
              "\"solve_before_setup_reason\": %d, \"pass\": %s}\n",
              ok1 ? "true" : "false", code1, msg1.c_str(), rel1, rel_err, solver.getStats().numIterations,
              ok2 ? "true" : "false", rel2, reason, pass ? "true" : "false");
  return pass ? 0 : 1;
}
