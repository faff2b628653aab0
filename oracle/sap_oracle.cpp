// ORACLE — test infrastructure, NOT product code.
//
// A CPU restatement of the SaP SPIKE-preconditioned BiCGStab(L) solve of
// spikegpu/SaPLibrary, used only as the checker of the CUDA product path
// (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg).  The
// product library never links, loads or calls this file.
//
// Parity pinning: the reference ships no golden vectors for this path (its
// single test is examples/unit_test/driver_unit_test.cu:49-94, a convergence
// assertion).  This restatement is pinned against that test's assertions and
// against the reference's own operation order, cited per function below.
// Every citation is relative to the reference project root.
//
// Layouts restated from the reference:
//  * band: column-major, 2K+1 entries per column; element (i,j) lives at
//    j*(2K+1) + K + (i-j)  (sap/device/data_transfer.cuh:423-448);
//  * partitions: P parts, the first N%P have N/P+1 rows
//    (sap/device/sweep_band_const.cuh:154-166);
//  * row-major input band (sap/banded_matrix.h:66-92): element (i,j) at
//    i*(2K+1) + K + (j-i).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <queue>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static const float kBurstValue = 1e-7f;     // sap/common.h:46
static const float kBurstNewValue = 1e-4f;  // sap/common.h:47
static const int kCriticalThreshold = 70;   // sap/common.h:66

enum { LU_UL = 0, LU_only = 1 };             // sap/common.h:86-89
enum { Spike = 0, Block = 1, NoPrecond = 2 };  // sap/common.h:94-98

struct Parts {
  int n = 0, P = 1, q = 0, r = 0;
  void init(int n_, int P_) { n = n_; P = P_; q = n / P; r = n % P; }
  int start(int p) const { return p * q + std::min(p, r); }
  int size(int p) const { return q + (p < r ? 1 : 0); }
};

// boostValue (sap/device/factor_band_const.cuh:17-40, 4-arg form).
template <typename T>
static inline T boost(T v) {
  if (v > (T)kBurstValue || v < -(T)kBurstValue) return v;
  return v < 0 ? -(T)kBurstNewValue : (T)kBurstNewValue;
}

template <typename T>
struct Precond {
  // options
  int P_req = 1, fact = LU_UL, ptype = Spike;
  bool safe = false;
  // state
  int n = 0, K = 0, P = 1;
  Parts parts;
  std::vector<T> B;      // factors, column-major band
  std::vector<T> offd;   // per interface i: B_i (KxK row-major) then C_{i+1}
  std::vector<T> V, W;   // per interface, KxK row-major tips
  std::vector<T> S;      // per interface, LU of I - W V (row-major), U rows post-divided
  int status = 0;
  std::string msg;
  // timing (ms) of the last setup
  double t_setup = 0;

  T& at(int i, int j) { return B[(size_t)j * (2 * K + 1) + K + (i - j)]; }
  T atc(int i, int j) const { return B[(size_t)j * (2 * K + 1) + K + (i - j)]; }
};

// ---------------------------------------------------------------------------
// Factorisations of one partition [s, e) in place on the band.
// bandLU_g32 / blockedBandLU_critical_const_phase1_safe
// (sap/device/factor_band_const.cuh:229-305, 1423-1483): pivot by pivot,
// divide the L column, then the rank-1 update of the (w x w) window.
template <typename T>
static void lu_partition(Precond<T>& pc, int s, int e, bool do_boost) {
  const int K = pc.K;
  for (int j = s; j < e; j++) {
    int w = std::min(K, e - 1 - j);
    T piv = pc.at(j, j);
    if (do_boost) { piv = boost(piv); pc.at(j, j) = piv; }
    for (int r = 1; r <= w; r++) pc.at(j + r, j) /= piv;
    for (int c = 1; c <= w; c++) {
      T u = pc.at(j, j + c);
      for (int r = 1; r <= w; r++) pc.at(j + r, j + c) -= pc.at(j + r, j) * u;
    }
  }
}

// bandUL_g32 / blockedBandUL_critical_const_phase1_safe
// (sap/device/factor_band_const.cuh:400-466, 1568-1628): mirror image, from
// the last row upward; U' is unit upper (multipliers above the diagonal).
template <typename T>
static void ul_partition(Precond<T>& pc, int s, int e, bool do_boost) {
  const int K = pc.K;
  for (int j = e - 1; j >= s; j--) {
    int w = std::min(K, j - s);
    T piv = pc.at(j, j);
    if (do_boost) { piv = boost(piv); pc.at(j, j) = piv; }
    for (int r = 1; r <= w; r++) pc.at(j - r, j) /= piv;
    for (int c = 1; c <= w; c++) {
      T l = pc.at(j, j - c);
      for (int r = 1; r <= w; r++) pc.at(j - r, j - c) -= pc.at(j - r, j) * l;
    }
  }
}

// hasZeroPivots (sap/precond.h:6337-6350): any |diag| < BURST_VALUE.
template <typename T>
static bool has_zero_pivot(const Precond<T>& pc, int s, int e) {
  for (int j = s; j < e; j++)
    if (std::fabs(pc.atc(j, j)) < kBurstValue) return true;
  return false;
}

// bandLU_post_divide / bandLUUL_post_divide
// (sap/device/factor_band_const.cuh:1717-1779): scale U rows (LU form) or
// L' rows (UL form) to a unit diagonal, restricted to the partition.
template <typename T>
static void post_divide_lu(Precond<T>& pc, int s, int e) {
  const int K = pc.K;
  for (int i = s; i < e; i++) {
    T d = pc.at(i, i);
    for (int j = i + 1; j <= std::min(e - 1, i + K); j++) pc.at(i, j) /= d;
  }
}
template <typename T>
static void post_divide_ul(Precond<T>& pc, int s, int e) {
  const int K = pc.K;
  for (int i = s; i < e; i++) {
    T d = pc.at(i, i);
    for (int j = std::max(s, i - K); j < i; j++) pc.at(i, j) /= d;
  }
}

// ---------------------------------------------------------------------------
// Sweeps over one partition (column oriented, sap/device/sweep_band_const.cuh:
// 1004-1275 for the LU_UL form, 248-312 / 535-584 for the LU form).
template <typename T>
static void sweep_partition(const Precond<T>& pc, T* g, int s, int e, bool ul_form) {
  const int K = pc.K;
  auto A = [&](int i, int j) { return pc.atc(i, j); };
  if (!ul_form) {
    for (int j = s; j < e - 1; j++) {
      int w = std::min(K, e - 1 - j);
      T gj = g[j];
      for (int t = 1; t <= w; t++) g[j + t] -= gj * A(j + t, j);
    }
    for (int j = s; j < e; j++) g[j] /= A(j, j);  // preBck divide (precond.h:5152-5155)
    for (int j = e - 1; j > s; j--) {
      int w = std::min(K, j - s);
      T gj = g[j];
      for (int t = 1; t <= w; t++) g[j - t] -= gj * A(j - t, j);
    }
  } else {
    for (int j = e - 1; j > s; j--) {
      int w = std::min(K, j - s);
      T gj = g[j];
      for (int t = 1; t <= w; t++) g[j - t] -= gj * A(j - t, j);
    }
    for (int j = s; j < e; j++) g[j] /= A(j, j);
    for (int j = s; j < e - 1; j++) {
      int w = std::min(K, e - 1 - j);
      T gj = g[j];
      for (int t = 1; t <= w; t++) g[j + t] -= gj * A(j + t, j);
    }
  }
}

template <typename T>
static void sweeps(const Precond<T>& pc, T* g) {
  const bool lu_ul = (pc.fact == LU_UL && pc.ptype == Spike && pc.P > 1);
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < pc.P; p++) {
    int s = pc.parts.start(p), e = s + pc.parts.size(p);
    sweep_partition(pc, g, s, e, lu_ul && p == pc.P - 1);
  }
}

// ---------------------------------------------------------------------------
// Dense LU of the Schur block S = I - W V without pivoting
// (fullLU_sub_spec + blockedFullLU_phase1..3 + fullLU_post_divide,
// sap/device/factor_band_var.cuh:736-800, 964-1107).
template <typename T>
static void dense_lu(T* S, int K, bool do_boost) {
  for (int j = 0; j < K; j++) {
    T piv = S[j * K + j];
    if (do_boost) { piv = boost(piv); S[j * K + j] = piv; }
    for (int r = j + 1; r < K; r++) S[r * K + j] /= piv;
    for (int r = j + 1; r < K; r++) {
      T l = S[r * K + j];
      for (int c = j + 1; c < K; c++) S[r * K + c] -= l * S[j * K + c];
    }
  }
  for (int r = 0; r < K; r++) {
    T d = S[r * K + r];
    for (int c = r + 1; c < K; c++) S[r * K + c] /= d;
  }
}

// Spike tips of the LU_UL method (calculateSpikes(B2,WV), sap/precond.h:
// 6232-6287; forwardElimLdWV / backwardElimUdWV, sweep_band_const.cuh:585-706).
// V_i = U_bb^-1 L_bb^-1 B_i from the LU corner of partition i;
// W_{i+1} = L'_tt^-1 U'_tt^-1 C_{i+1} from the UL corner of partition i+1.
template <typename T>
static void spikes_lu_ul(Precond<T>& pc, const Precond<T>& lu, const Precond<T>& ul) {
  const int K = pc.K, P = pc.P;
  pc.V.assign((size_t)(P - 1) * K * K, 0.f);
  pc.W.assign((size_t)(P - 1) * K * K, 0.f);
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < P - 1; i++) {
    int s = pc.parts.start(i + 1);
    const T* Bi = &pc.offd[(size_t)(2 * i) * K * K];
    const T* Ci = &pc.offd[(size_t)(2 * i + 1) * K * K];
    T* Vi = &pc.V[(size_t)i * K * K];
    T* Wi = &pc.W[(size_t)i * K * K];
    std::vector<T> x(K);
    for (int col = 0; col < K; col++) {
      // V column `col`
      for (int r = 0; r < K; r++) x[r] = Bi[r * K + col];
      int base = s - K;
      for (int j = 0; j < K - 1; j++)
        for (int t = 1; t < K - j; t++) x[j + t] -= x[j] * lu.atc(base + j + t, base + j);
      for (int j = K - 1; j >= 0; j--) {
        x[j] /= lu.atc(base + j, base + j);
        for (int t = 1; t <= j; t++) x[j - t] -= x[j] * lu.atc(base + j - t, base + j);
      }
      for (int r = 0; r < K; r++) Vi[r * K + col] = x[r];
      // W column `col`
      for (int r = 0; r < K; r++) x[r] = Ci[r * K + col];
      base = s;
      for (int j = K - 1; j >= 0; j--)
        for (int t = 1; t <= j; t++) x[j - t] -= x[j] * ul.atc(base + j - t, base + j);
      for (int j = 0; j < K; j++) {
        x[j] /= ul.atc(base + j, base + j);
        for (int t = 1; t < K - j; t++) x[j + t] -= x[j] * ul.atc(base + j + t, base + j);
      }
      for (int r = 0; r < K; r++) Wi[r * K + col] = x[r];
    }
  }
}

// Spike tips for the const-band LU_only method: V as above, W from a full
// forward sweep of partition i+1 with K right-hand sides followed by a full
// backward sweep (calculateSpikes_const, sap/precond.h:5785-5949).  The
// reference never post-divides U in this mode while its backward sweep
// assumes it (documented deviation): here U is used consistently.
template <typename T>
static void spikes_lu_only(Precond<T>& pc) {
  const int K = pc.K, P = pc.P;
  pc.V.assign((size_t)(P - 1) * K * K, 0.f);
  pc.W.assign((size_t)(P - 1) * K * K, 0.f);
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < P - 1; i++) {
    int s = pc.parts.start(i + 1);
    int e = s + pc.parts.size(i + 1);
    const T* Bi = &pc.offd[(size_t)(2 * i) * K * K];
    const T* Ci = &pc.offd[(size_t)(2 * i + 1) * K * K];
    T* Vi = &pc.V[(size_t)i * K * K];
    T* Wi = &pc.W[(size_t)i * K * K];
    std::vector<T> x(K);
    for (int col = 0; col < K; col++) {
      for (int r = 0; r < K; r++) x[r] = Bi[r * K + col];
      int base = s - K;
      for (int j = 0; j < K - 1; j++)
        for (int t = 1; t < K - j; t++) x[j + t] -= x[j] * pc.atc(base + j + t, base + j);
      for (int j = K - 1; j >= 0; j--) {
        x[j] /= pc.atc(base + j, base + j);
        for (int t = 1; t <= j; t++) x[j - t] -= x[j] * pc.atc(base + j - t, base + j);
      }
      for (int r = 0; r < K; r++) Vi[r * K + col] = x[r];
      // full sweeps of partition i+1 (U not yet post-divided here)
      int np = e - s;
      std::vector<T> y(np, 0.f);
      for (int r = 0; r < K; r++) y[r] = Ci[r * K + col];
      for (int j = 0; j < np - 1; j++) {
        int w = std::min(K, np - 1 - j);
        T yj = y[j];
        if (yj == 0.f) continue;
        for (int t = 1; t <= w; t++) y[j + t] -= yj * pc.atc(s + j + t, s + j);
      }
      for (int j = np - 1; j >= 0; j--) {
        y[j] /= pc.atc(s + j, s + j);
        int w = std::min(K, j);
        T yj = y[j];
        for (int t = 1; t <= w; t++) y[j - t] -= yj * pc.atc(s + j - t, s + j);
      }
      for (int r = 0; r < K; r++) Wi[r * K + col] = y[r];
    }
  }
}

// extractOffDiagonal / copydWV (sap/precond.h:2371-2400,
// sap/device/data_transfer.cuh:129-199).
template <typename T>
static void extract_offdiag(Precond<T>& pc) {
  const int K = pc.K, P = pc.P;
  pc.offd.assign((size_t)2 * (P - 1) * K * K, 0.f);
  for (int i = 0; i < P - 1; i++) {
    int s = pc.parts.start(i + 1);
    T* Bi = &pc.offd[(size_t)(2 * i) * K * K];
    T* Ci = &pc.offd[(size_t)(2 * i + 1) * K * K];
    for (int c = 0; c < K; c++)
      for (int r = 0; r < K; r++) {
        Bi[c * K + r] = (r > c) ? 0.f : pc.at(s - K + c, s + r);
        Ci[c * K + r] = (c > r) ? 0.f : pc.at(s + c, s - K + r);
      }
  }
}

// Reduced matrix R_i = [[I, V_i], [W_i, I]] and its LU: first K pivots are
// one, the trailing block is S = I - W V (assembleReducedMat + partFullLU,
// sap/precond.h:2412-2429, 2549-2611, 6292-6320).
template <typename T>
static void reduced_factor(Precond<T>& pc) {
  const int K = pc.K, P = pc.P;
  pc.S.assign((size_t)(P - 1) * K * K, 0.f);
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < P - 1; i++) {
    const T* Vi = &pc.V[(size_t)i * K * K];
    const T* Wi = &pc.W[(size_t)i * K * K];
    T* Si = &pc.S[(size_t)i * K * K];
    for (int c = 0; c < K; c++)
      for (int r = 0; r < K; r++) {
        T t = (c == r) ? 1.f : 0.f;
        for (int cur = 0; cur < K; cur++) t -= Wi[c * K + cur] * Vi[cur * K + r];
        Si[c * K + r] = t;
      }
    dense_lu(Si, K, pc.safe);
  }
}

// Setup for a constant-bandwidth matrix already in the column-major band
// (Precond::setup, sap/precond.h:910-1362, LU_UL branch 1296-1350, LU_only
// branch 1268-1294, single partition / Block 1215-1238).
template <typename T>
static void setup_band(Precond<T>& pc) {
  const int K = pc.K;
  pc.status = 0;
  pc.msg.clear();
  if (pc.ptype == NoPrecond) return;
  if (K == 0) return;
  pc.parts.init(pc.n, pc.P);
  if (pc.ptype == Block || pc.P == 1) {
    // partBlockedBandedLU_one boosts only in safe mode (precond.h:3995-4070);
    // the multi-partition const kernels for K >= 70 always boost.
    bool bst = pc.safe || (pc.P > 1 && K >= kCriticalThreshold);
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < pc.P; p++) {
      int s = pc.parts.start(p);
      lu_partition(pc, s, s + pc.parts.size(p), bst);
    }
    if (!pc.safe && has_zero_pivot(pc, 0, pc.n)) {
      pc.status = -1; pc.msg = "Found a pivot equal to zero"; return;
    }
    for (int p = 0; p < pc.P; p++) {
      int s = pc.parts.start(p);
      post_divide_lu(pc, s, s + pc.parts.size(p));
    }
    return;
  }
  extract_offdiag(pc);
  bool bst = pc.safe || K >= kCriticalThreshold;
  if (pc.fact == LU_UL) {
    Precond<T> ul = pc;  // B2 = m_B
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < 2 * (pc.P - 1); p++) {
      if (p < pc.P - 1) {
        int s = pc.parts.start(p);
        lu_partition(pc, s, s + pc.parts.size(p), bst);
      } else {
        int q = p - (pc.P - 1) + 1;
        int s = pc.parts.start(q);
        ul_partition(ul, s, s + pc.parts.size(q), bst);
      }
    }
    int lastS = pc.parts.start(pc.P - 1);
    if (!pc.safe && (has_zero_pivot(pc, 0, lastS) ||
                     has_zero_pivot(ul, pc.parts.start(1), pc.n))) {
      pc.status = -1; pc.msg = "Found a pivot equal to zero"; return;
    }
    spikes_lu_ul(pc, pc, ul);
    // copyLastPartition (precond.h:6326-6330)
    std::copy(ul.B.begin() + (size_t)(2 * K + 1) * lastS, ul.B.end(),
              pc.B.begin() + (size_t)(2 * K + 1) * lastS);
    for (int p = 0; p < pc.P - 1; p++) {
      int s = pc.parts.start(p);
      post_divide_lu(pc, s, s + pc.parts.size(p));
    }
    post_divide_ul(pc, lastS, pc.n);
  } else {
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < pc.P; p++) {
      int s = pc.parts.start(p);
      lu_partition(pc, s, s + pc.parts.size(p), bst);
    }
    if (!pc.safe && has_zero_pivot(pc, 0, pc.n)) {
      pc.status = -1; pc.msg = "Found a pivot equal to zero"; return;
    }
    spikes_lu_only(pc);
    for (int p = 0; p < pc.P; p++) {
      int s = pc.parts.start(p);
      post_divide_lu(pc, s, s + pc.parts.size(p));
    }
  }
  reduced_factor(pc);
}

// Preconditioner apply z = M^-1 v (Precond::operator() + solve + getSRev,
// sap/precond.h:1370-1528): two partitioned sweep pairs around the
// truncated reduced solve (partFullFwdSweep/BckSweep 5418-5487) and the
// purification of the interface right-hand sides (purifyRHS 5494-5530).
template <typename T>
static void apply(const Precond<T>& pc, const double* v, double* z) {
  const int n = pc.n, K = pc.K, P = pc.P;
  if (pc.ptype == NoPrecond) { std::copy(v, v + n, z); return; }
  std::vector<T> f(n), g(n);
  for (int i = 0; i < n; i++) f[i] = (T)v[i];
  if (K == 0) {
    for (int i = 0; i < n; i++) z[i] = (double)(f[i] / pc.B[i]);
    return;
  }
  if (P > 1 && pc.ptype == Spike) {
    g = f;
    sweeps(pc, g.data());
    for (int i = 0; i < P - 1; i++) {
      int s = pc.parts.start(i + 1);
      const T* Vi = &pc.V[(size_t)i * K * K];
      const T* Wi = &pc.W[(size_t)i * K * K];
      const T* Si = &pc.S[(size_t)i * K * K];
      T* xb = &g[s - K];
      T* xt = &g[s];
      std::vector<T> z2(K);
      for (int r = 0; r < K; r++) {
        T t = xt[r];
        for (int c = 0; c < K; c++) t -= Wi[r * K + c] * xb[c];
        z2[r] = t;
      }
      for (int r = 0; r < K; r++)
        for (int c = 0; c < r; c++) z2[r] -= Si[r * K + c] * z2[c];
      for (int r = 0; r < K; r++) z2[r] /= Si[r * K + r];
      for (int r = K - 1; r >= 0; r--)
        for (int c = r + 1; c < K; c++) z2[r] -= Si[r * K + c] * z2[c];
      for (int r = 0; r < K; r++) {
        T t = xb[r];
        for (int c = 0; c < K; c++) t -= Vi[r * K + c] * z2[c];
        xb[r] = t;
      }
      for (int r = 0; r < K; r++) xt[r] = z2[r];
    }
    for (int i = 0; i < P - 1; i++) {
      int s = pc.parts.start(i + 1);
      const T* Bi = &pc.offd[(size_t)(2 * i) * K * K];
      const T* Ci = &pc.offd[(size_t)(2 * i + 1) * K * K];
      for (int c = 0; c < K; c++) {
        T t1 = 0.f, t2 = 0.f;
        for (int r = 0; r < K; r++) {
          t1 += Bi[c * K + r] * g[s + r];
          t2 += Ci[c * K + r] * g[s - K + r];
        }
        f[s - K + c] -= t1;
        f[s + c] -= t2;
      }
    }
  }
  sweeps(pc, f.data());
  for (int i = 0; i < n; i++) z[i] = (double)f[i];
}

// ---------------------------------------------------------------------------
// SpMV (FP64).  MVBanded (sap/spmv.h:27-74, matrix_multiply.cuh:301-350) and
// the CSR product SpmvCusp delegates to (sap/spmv.h:110-121).
struct Op {
  int n = 0;
  int K = 0;
  const double* band = nullptr;  // row-major band
  const int* rp = nullptr;
  const int* ci = nullptr;
  const double* vals = nullptr;
  void apply(const double* x, double* y) const {
    if (band) {
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) {
        int lo = std::max(0, i - K), hi = std::min(n - 1, i + K);
        double t = 0;
        const double* row = band + (size_t)i * (2 * K + 1) + K - i;
        for (int j = lo; j <= hi; j++) t += row[j] * x[j];
        y[i] = t;
      }
    } else {
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) {
        double t = 0;
        for (int p = rp[i]; p < rp[i + 1]; p++) t += vals[p] * x[ci[p]];
        y[i] = t;
      }
    }
  }
};

static double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  const int n = (int)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}
static double nrm2(const std::vector<double>& a) { return std::sqrt(dot(a, a)); }
static void axpy(const std::vector<double>& x, std::vector<double>& y, double a) {
  const int n = (int)x.size();
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) y[i] += a * x[i];
}
// z = a x + b y
static void axpby(const std::vector<double>& x, const std::vector<double>& y,
                  std::vector<double>& z, double a, double b) {
  const int n = (int)x.size();
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) z[i] = a * x[i] + b * y[i];
}

// BiCGStabLMonitor (sap/monitor.h:154-339).
struct Monitor {
  int maxIt = 100, maxm = 8, stag = 0, more = 0, maxStag = 3;
  double relTol = 1e-6, absTol = 0, rhsNorm = 0, rNorm = std::numeric_limits<double>::max();
  float it = 0;
  int code = 0;
  std::string msg;
  double tol() const { return absTol + relTol * rhsNorm; }
  void stop(int c, const char* m) { code = c; msg = m; }
  bool finished(double r) {
    rNorm = r;
    if (code != 0) return true;
    if (std::isnan(rNorm)) stop(-2, "Residual norm is NaN");
    else if (rNorm <= tol()) stop(1, "Converged");
    else if (it > maxIt) stop(-1, "Maximum number of iterations was reached");
    else {
      if (stag >= maxStag && more == 0) stag = 0;
      more++;
      if (more >= maxm) stop(-3, "Stagnation encountered");
    }
    return code != 0;
  }
  bool finished() {
    if (code != 0) return true;
    if (it > maxIt) stop(-1, "Maximum number of iterations was reached");
    return code != 0;
  }
  bool needCheck(double r) {
    rNorm = r;
    if (code != 0) return false;
    if (std::isnan(rNorm)) stop(-2, "Residual norm is NaN");
    return code == 0 && (rNorm <= tol() || stag >= maxStag || more);
  }
};

using Apply = std::function<void(const std::vector<double>&, std::vector<double>&)>;

// Monitor::finished (sap/monitor.h:134-149), the default monitor of the
// BiCGStab and MINRES drivers.
static bool finished_default(Monitor& mon, double r) {
  mon.rNorm = r;
  if (mon.code != 0) return true;
  if (std::isnan(mon.rNorm)) mon.stop(-2, "Residual norm is NaN");
  else if (mon.rNorm <= mon.tol()) mon.stop(1, "Converged");
  else if (mon.it > mon.maxIt) mon.stop(-1, "Maximum number of iterations was reached");
  return mon.code != 0;
}

// cusp::blas::axpbypcz: out = a x + b y + c z
static void axpbypcz(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z,
                     std::vector<double>& out, double a, double b, double c) {
  for (size_t i = 0; i < out.size(); i++) out[i] = a * x[i] + b * y[i] + c * z[i];
}

// sap::bicgstab (sap/bicgstab.h:50-155), restated line by line.
static void bicgstab_classic(const Apply& A, const Apply& M, std::vector<double>& x, const std::vector<double>& b,
                             Monitor& mon) {
  const size_t N = b.size();
  std::vector<double> y(N), p(N), r(N), r_star(N), s(N), Mp(N), AMp(N), Ms(N), AMs(N);
  A(x, y);
  axpby(b, y, r, 1.0, -1.0);
  p = r;
  r_star = r;
  double r_r_star_old = dot(r_star, r);
  while (!finished_default(mon, nrm2(r))) {
    if (r_r_star_old == 0) { mon.stop(-10, "r_r_star is zero"); break; }
    M(p, Mp);
    A(Mp, AMp);
    const double tmp1 = dot(r_star, AMp);
    if (tmp1 == 0) { mon.stop(-11, "r_star * AMp is zero"); break; }
    const double alpha = r_r_star_old / tmp1;
    axpby(r, AMp, s, 1.0, -alpha);
    if (finished_default(mon, nrm2(s))) {
      axpby(x, Mp, x, 1.0, alpha);
      break;
    }
    M(s, Ms);
    A(Ms, AMs);
    const double tmp2 = dot(AMs, AMs);
    if (tmp2 == 0) { mon.stop(-12, "AMs * AMs is zero"); break; }
    const double omega = dot(AMs, s) / tmp2;
    axpbypcz(x, Mp, Ms, x, 1.0, alpha, omega);
    axpby(s, AMs, r, 1.0, -omega);
    const double r_r_star_new = dot(r_star, r);
    const double beta = (r_r_star_new / r_r_star_old) * (alpha / omega);
    r_r_star_old = r_r_star_new;
    axpbypcz(r, p, AMp, p, 1.0, beta, -beta * omega);
    mon.it += 1.f;
  }
}

// sap::minres (sap/minres.h:40-195), restated line by line.
static void minres(const Apply& A, const Apply& P, std::vector<double>& x, const std::vector<double>& b,
                   Monitor& mon) {
  const double eps = std::numeric_limits<double>::epsilon();
  const size_t n = b.size();
  auto count = [&]() { return (size_t)(mon.it + 0.5f); };
  std::vector<double> y(n), r1(n);
  A(x, r1);
  axpby(b, r1, r1, 1.0, -1.0);
  P(r1, y);
  double beta1 = dot(r1, y);
  if (beta1 < 0) {
    mon.stop(-10, "The preconditioner is not positive definite");
    beta1 *= -1;
  } else if (beta1 > 0) {
    beta1 = std::sqrt(beta1);
  }
  double Anorm = 0, ynorm = 0, phibar = beta1;
  double oldb = 0, beta = beta1, dbar = 0, epsln = 0, oldeps = 0;
  double phi = 0, rhs1 = beta1, rhs2 = 0, tnorm2 = 0;
  double cs = -1, sn = 0, gmax = 0, gmin = std::numeric_limits<double>::max();
  double alpha = 0, gamma = 0, delta = 0, gbar = 0, z = 0;
  std::vector<double> v(n), w(n, 0.0), w1(n, 0.0), w2(n, 0.0), r2 = r1;
  while (!finished_default(mon, phibar)) {
    const double s = 1 / beta;
    for (size_t i = 0; i < n; i++) v[i] = y[i] * s;
    A(v, y);
    if (count() > 0) axpby(y, r1, y, 1.0, -beta / oldb);
    alpha = dot(v, y);
    axpby(y, r2, y, 1.0, -alpha / beta);
    r1 = r2;
    r2 = y;
    P(r2, y);
    oldb = beta;
    beta = dot(r2, y);
    if (beta < 0) { mon.stop(-10, "The preconditioner is not positive definite"); break; }
    beta = std::sqrt(beta);
    tnorm2 += alpha * alpha + oldb * oldb + beta * beta;
    if (count() == 0 && beta / beta1 <= 10 * eps) mon.stop(10, "beta2 = 0. If M = I, b and x are eigenvectors");
    oldeps = epsln;
    delta = cs * dbar + sn * alpha;
    gbar = sn * dbar - cs * alpha;
    epsln = sn * beta;
    dbar = -cs * beta;
    const double root = std::sqrt(gbar * gbar + dbar * dbar);
    gamma = std::sqrt(gbar * gbar + beta * beta);
    gamma = std::max(gamma, eps);
    cs = gbar / gamma;
    sn = beta / gamma;
    phi = cs * phibar;
    phibar = sn * phibar;
    const double denom = 1 / gamma;
    w1 = w2;
    w2 = w;
    axpbypcz(v, w1, w2, w, denom, -oldeps * denom, -delta * denom);
    axpby(x, w, x, 1.0, phi);
    gmax = std::max(gmax, gamma);
    gmin = std::min(gmin, gamma);
    z = rhs1 / gamma;
    rhs1 = rhs2 - delta * z;
    rhs2 = -epsln * z;
    Anorm = std::sqrt(tnorm2);
    ynorm = nrm2(x);
    if (mon.code != 10) {
      const double test2 = root / Anorm, Acond = gmax / gmin;
      if (Acond >= 0.1 / eps) mon.stop(11, "x has converged to an eigenvector");
      if (Anorm * eps * ynorm >= beta1) mon.stop(12, "Reasonable accuracy achieved, given eps");
      if (test2 <= mon.absTol) mon.stop(13, "A least-squares solution was found, given tol");
    }
    mon.it += 1.f;
  }
}

// bicgstabl<..., L> (sap/bicgstab2.h:32-360), restated line by line.
static void bicgstabl(const Apply& A, const Apply& P, std::vector<double>& x,
                      const std::vector<double>& b, Monitor& mon, int L) {
  const int n = (int)b.size();
  const double eps = 1e-20;
  double rho0 = 1, alpha = 0, omega = 1, rho1;
  std::vector<double> r0(n), r(n), u(n, 0.0), xx(n), Pv(n);
  std::vector<std::vector<double>> rr(L + 1, std::vector<double>(n, 0.0)),
      uu(L + 1, std::vector<double>(n, 0.0));
  std::vector<std::vector<double>> tao(L + 1, std::vector<double>(L + 1, 0.0));
  std::vector<double> gamma(L + 2), gp(L + 2), gpp(L + 2), sigma(L + 2);
  A(x, r0);
  axpby(b, r0, r0, 1.0, -1.0);
  r = r0;
  uu[0] = u; xx = x; rr[0] = r;
  double r_norm_min = nrm2(r), r_norm = r_norm_min, r_norm_act = r_norm;
  std::vector<double> x_min(n, 0.0), Pxx(n), APxx(n);
  auto recheck = [&]() {
    P(xx, Pxx);
    A(Pxx, APxx);
    axpby(b, APxx, rr[0], 1.0, -1.0);
    r_norm_act = nrm2(rr[0]);
  };
  while (true) {
    rho0 = -omega * rho0;
    mon.it += 0.25f;
    for (int j = 0; j < L; j++) {
      rho1 = dot(rr[j], r0);
      if (rho0 == 0) { mon.stop(-10, "rho0 is zero"); break; }
      double beta = alpha * rho1 / rho0;
      rho0 = rho1;
      for (int i = 0; i <= j; i++) axpby(rr[i], uu[i], uu[i], 1.0, -beta);
      P(uu[j], Pv);
      A(Pv, uu[j + 1]);
      double gam = dot(uu[j + 1], r0);
      if (gam == 0) { mon.stop(-11, "gamma is zero"); break; }
      alpha = rho0 / gam;
      for (int i = 0; i <= j; i++) axpy(uu[i + 1], rr[i], -alpha);
      r_norm_act = r_norm = nrm2(rr[0]);
      P(rr[j], Pv);
      A(Pv, rr[j + 1]);
      if (std::fabs(alpha) * nrm2(uu[0]) < eps * nrm2(xx)) mon.stag++;
      else mon.stag = 0;
      axpy(uu[0], xx, alpha);
      if (mon.needCheck(r_norm)) {
        recheck();
        if (mon.finished(r_norm_act)) break;
      }
      if (r_norm_act < r_norm_min) { r_norm_min = r_norm_act; x_min = xx; }
      if (mon.finished()) break;
    }
    if (mon.finished()) break;
    for (int j = 1; j <= L; j++) {
      for (int i = 1; i < j; i++) {
        tao[i][j] = dot(rr[j], rr[i]) / sigma[i];
        axpy(rr[i], rr[j], -tao[i][j]);
      }
      sigma[j] = dot(rr[j], rr[j]);
      if (sigma[j] == 0) { mon.stop(-12, "a sigma value is zero"); break; }
      gp[j] = dot(rr[j], rr[0]) / sigma[j];
    }
    if (mon.finished()) break;
    gamma[L] = gp[L];
    omega = gamma[L];
    for (int j = L - 1; j > 0; j--) {
      gamma[j] = gp[j];
      for (int i = j + 1; i <= L; i++) gamma[j] -= tao[j][i] * gamma[i];
    }
    for (int j = 1; j < L; j++) {
      gpp[j] = gamma[j + 1];
      for (int i = j + 1; i < L; i++) gpp[j] += tao[j][i] * gamma[i + 1];
    }
    if (std::fabs(gamma[1]) * nrm2(rr[0]) < eps * nrm2(xx)) mon.stag++;
    else mon.stag = 0;
    axpy(rr[0], xx, gamma[1]);
    axpy(rr[L], rr[0], -gp[L]);
    axpy(uu[L], uu[0], -gamma[L]);
    r_norm_act = r_norm = nrm2(rr[0]);
    mon.it += 0.25f;
    if (mon.needCheck(r_norm)) {
      recheck();
      if (mon.finished(r_norm_act)) break;
    }
    if (r_norm_act < r_norm_min) { r_norm_min = r_norm_act; x_min = xx; }
    if (mon.finished()) break;
    mon.it += 0.25f;
    bool brk = false;
    for (int j = 1; j < L; j++) {
      axpy(uu[j], uu[0], -gamma[j]);
      if (std::fabs(gpp[j]) * nrm2(rr[j]) < eps * nrm2(xx)) mon.stag++;
      else mon.stag = 0;
      axpy(rr[j], xx, gpp[j]);
      axpy(rr[j], rr[0], -gp[j]);
      r_norm_act = r_norm = nrm2(rr[0]);
      if (mon.needCheck(r_norm)) {
        recheck();
        if (mon.finished(r_norm_act)) { brk = true; break; }
      }
      if (r_norm_act < r_norm_min) { r_norm_min = r_norm_act; x_min = xx; }
      if (mon.finished()) { brk = true; break; }
    }
    (void)brk;
    if (mon.finished()) break;
    u = uu[0]; x = xx; r = rr[0];
    mon.it += 0.25f;
  }
  if (mon.code > 0) {
    P(xx, x);
  } else {
    std::vector<double> Pxmin(n), APxmin(n), rc(n), rcm(n);
    P(xx, Pxx);
    A(Pxx, APxx);
    axpby(b, APxx, rc, 1.0, -1.0);
    P(x_min, Pxmin);
    A(Pxmin, APxmin);
    axpby(b, APxmin, rcm, 1.0, -1.0);
    double a = nrm2(rc), c = nrm2(rcm);
    if (a < c) { x = Pxx; mon.rNorm = a; }
    else { x = Pxmin; mon.rNorm = c; }
  }
}

}  // namespace orc

// ---------------------------------------------------------------------------
// C entry points used through ctypes by the tests and the bench's CPU leg.
namespace orc {
// A preconditioner of either precision (the Solver's PrecValueType,
// sap/solver.h:153).
struct Handle {
  int dtype = 0;  // 0 float, 1 double
  Precond<float> f;
  Precond<double> d;
  template <typename Fn> auto visit(Fn fn) { return dtype ? fn(d) : fn(f); }
};

template <typename T>
static void setup_from_rowmajor(Precond<T>& pc, int n, int K, const double* band_rm) {
  pc.n = n; pc.K = K;
  int maxP = std::max(1, n / std::max(K + 1, 2 * K));
  pc.P = std::min(pc.P_req, maxP);
  pc.B.assign((size_t)(2 * K + 1) * n, T(0));
  for (int i = 0; i < n; i++)
    for (int j = std::max(0, i - K); j <= std::min(n - 1, i + K); j++)
      pc.at(i, j) = (T)band_rm[(size_t)i * (2 * K + 1) + K + (j - i)];
  setup_band(pc);
}

template <typename T>
static void setup_from_csr(Precond<T>& pc, int n, const int* rp, const int* ci, const double* v) {
  pc.n = n;
  int K = 0;
  for (int i = 0; i < n; i++)
    for (int p = rp[i]; p < rp[i + 1]; p++) K = std::max(K, std::abs(i - ci[p]));
  pc.K = K;
  int maxP = std::max(1, n / std::max(K + 1, 2 * K));
  pc.P = std::min(pc.P_req, maxP);
  pc.B.assign((size_t)(2 * K + 1) * n, T(0));
  for (int i = 0; i < n; i++)
    for (int p = rp[i]; p < rp[i + 1]; p++) pc.at(i, ci[p]) = (T)v[p];
  setup_band(pc);
}
}  // namespace orc

extern "C" {

struct orc_result {
  int code;            // monitor code
  float iterations;    // 0.25-granular
  double rhs_norm;
  double res_norm;
  double rel_res_norm;
  int n, K, P;
  int status;          // setup status (sap::system_error::Reason or 0)
};

void* orc_precond_create(int P, int fact, int ptype, int safe, int dtype) {
  auto* h = new orc::Handle();
  h->dtype = dtype;
  h->visit([&](auto& pc) { pc.P_req = P; pc.fact = fact; pc.ptype = ptype; pc.safe = safe != 0; return 0; });
  return h;
}

void orc_precond_destroy(void* h) { delete (orc::Handle*)h; }

// CPU-baseline timing sample: the first `steps` pivots of the partition LU
// above (lu_partition, restating bandLU_g32) on a diagonally dominant band
// of half-bandwidth K (off-diagonals from a fixed LCG in [-1, 1], diagonal
// the row sum of their magnitudes), in FP64.  Returns the seconds of the
// pivots alone (band construction excluded).
double orc_band_lu_sample(int K, int steps) {
  orc::Precond<double> pc;
  pc.K = K;
  const int n = steps + K + 1;
  pc.n = n;
  pc.B.assign((size_t)(2 * K + 1) * n, 0.0);
  unsigned long long s = 0x9E3779B97F4A7C15ull;
  std::vector<double> rowsum(n, 0.0);
  for (int j = 0; j < n; j++)
    for (int i = std::max(0, j - K); i <= std::min(n - 1, j + K); i++) {
      if (i == j) continue;
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      const double v = (double)(s >> 11) / 9007199254740992.0 * 2.0 - 1.0;
      pc.at(i, j) = v;
      rowsum[i] += std::fabs(v);
    }
  for (int i = 0; i < n; i++) pc.at(i, i) = rowsum[i];
  const auto t0 = std::chrono::steady_clock::now();
  for (int j = 0; j < steps; j++) {
    const int w = std::min(K, n - 1 - j);
    const double piv = pc.at(j, j);
    for (int r = 1; r <= w; r++) pc.at(j + r, j) /= piv;
    for (int c = 1; c <= w; c++) {
      const double u = pc.at(j, j + c);
      for (int r = 1; r <= w; r++) pc.at(j + r, j + c) -= pc.at(j + r, j) * u;
    }
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// convertToBandedMatrix(BandedMatrix) (sap/precond.h:2103-2233).
int orc_setup_banded(void* h, int n, int K, const double* band_rm) {
  return ((orc::Handle*)h)->visit([&](auto& pc) { orc::setup_from_rowmajor(pc, n, K, band_rm); return pc.status; });
}

// convertToBandedMatrix(CSR) without reordering (sap/precond.h:2240-2368).
int orc_setup_csr(void* h, int n, const int* rp, const int* ci, const double* v) {
  return ((orc::Handle*)h)->visit([&](auto& pc) { orc::setup_from_csr(pc, n, rp, ci, v); return pc.status; });
}

void orc_info(void* h, int* n, int* K, int* P) {
  ((orc::Handle*)h)->visit([&](auto& pc) { *n = pc.n; *K = pc.K; *P = pc.P; return 0; });
}

void orc_apply(void* h, const double* v, double* z) {
  ((orc::Handle*)h)->visit([&](auto& pc) { orc::apply(pc, v, z); return 0; });
}

// Copies factor arrays out as doubles: 0 band, 1 V, 2 W, 3 S, 4 off-diagonals.
long long orc_factor_copy(void* h, int which, double* out) {
  return ((orc::Handle*)h)->visit([&](auto& pc) -> long long {
    const auto* vec = &pc.B;
    switch (which) {
      case 1: vec = &pc.V; break;
      case 2: vec = &pc.W; break;
      case 3: vec = &pc.S; break;
      case 4: vec = &pc.offd; break;
      default: break;
    }
    if (out)
      for (size_t i = 0; i < vec->size(); i++) out[i] = (double)(*vec)[i];
    return (long long)vec->size();
  });
}

void orc_spmv_banded(int n, int K, const double* band, const double* x, double* y) {
  orc::Op op; op.n = n; op.K = K; op.band = band; op.apply(x, y);
}
void orc_spmv_csr(int n, const int* rp, const int* ci, const double* v, const double* x, double* y) {
  orc::Op op; op.n = n; op.rp = rp; op.ci = ci; op.vals = v; op.apply(x, y);
}

// Full solve with a preconditioner set up beforehand, against a banded
// (band != NULL) or CSR operator (Solver::solve, sap/solver.h:477-562).
int orc_solve(void* h, int n, int K, const double* band, const int* rp, const int* ci,
              const double* vals, const double* b, double* x, int L, int maxit,
              double reltol, double abstol, orc_result* res) {
  auto* H = (orc::Handle*)h;
  orc::Op op; op.n = n; op.K = K; op.band = band; op.rp = rp; op.ci = ci; op.vals = vals;
  orc::Monitor mon; mon.maxIt = maxit; mon.relTol = reltol; mon.absTol = abstol;
  std::vector<double> bv(b, b + n), xv(x, x + n);
  mon.rhsNorm = orc::nrm2(bv);
  orc::Apply A = [&](const std::vector<double>& in, std::vector<double>& out) { op.apply(in.data(), out.data()); };
  orc::Apply Pm = [&](const std::vector<double>& in, std::vector<double>& out) {
    H->visit([&](auto& pc) { orc::apply(pc, in.data(), out.data()); return 0; });
  };
  // L >= 1: BiCGStab(L); L == 0: sap::bicgstab; L == -1: sap::minres
  if (L >= 1) orc::bicgstabl(A, Pm, xv, bv, mon, L);
  else if (L == 0) orc::bicgstab_classic(A, Pm, xv, bv, mon);
  else orc::minres(A, Pm, xv, bv, mon);
  std::copy(xv.begin(), xv.end(), x);
  res->code = mon.code; res->iterations = mon.it; res->rhs_norm = mon.rhsNorm;
  res->res_norm = mon.rNorm; res->rel_res_norm = mon.rNorm / mon.rhsNorm;
  H->visit([&](auto& pc) { res->n = pc.n; res->K = pc.K; res->P = pc.P; res->status = pc.status; return 0; });
  return mon.code;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
#include "reorder_oracle.cpp"
