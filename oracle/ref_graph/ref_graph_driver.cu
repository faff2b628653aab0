// ORACLE — test infrastructure only (never linked into, or loaded by, the
// product).  The reference's own reordering pipeline, sap/graph.h of
// spikegpu/SaPLibrary compiled unchanged from its source tree against the
// CUSP stand-in of this directory, driven as Precond::transformToBandedMatrix
// drives it (sap/precond.h:1656-1781 and the permutation composition of
// 2071-2089):
//   1. the CSR matrix in PrecValueType (float or double), explicit zeros removed
//      (precond.h:1667-1713; the input is sorted by row);
//   2. Graph<PrecValueType>::reorder: DB matching and scaling (with its device weight
//      kernel, sap/device/db.cuh), then RCM when maxBandwidth > 64
//      (precond.h:1735-1738);
//   3. Graph::dropOff when the band exceeds maxBandwidth or a drop-off
//      fraction is set (precond.h:1763-1775);
//   4. the partition clamp min(P, max(n / (K + 1), 1)) (precond.h:1777-1778);
//   5. for a variable band: assembleOffDiagMatrices, secondLevelReordering,
//      assembleBandedMatrix (precond.h:1785-1808);
//   6. combinePermutation (precond.h:1628-1636: finalPerm[i] = perm2[perm[i]])
//      applied as at precond.h:2071-2089.
// The graph.h calls need a GPU (DB's device vectors and kernel).  Built by
// oracle/ref_graph/build_ref.sh into oracle/_ref/libref_graph.so.
#include <cusp/shim.h>

#include <sap/graph.h>

#include <cstring>
#include <string>
#include <vector>

namespace {

struct RefResult {
  int n = 0, K = 0, P = 0, k_db = 0, k_reorder = 0, varBand = 0, status = 0;
  double drop_actual = 0;
  std::string msg;
  // same order as the oracle's integer outputs
  std::vector<int> ints[15];
};

template <typename A>
std::vector<int> to_std(const A& a) {
  thrust::host_vector<int> h(a.begin(), a.end());
  return std::vector<int>(h.begin(), h.end());
}

template <typename T>
void run(RefResult& r, int n, const int* rp, const int* ci, const double* v, int P_req, double dropFrac, int doDB,
         int scale, int maxBandwidth, int varBand) {
  typedef sap::Graph<T> G;
  // 1. PrecValueType CSR without explicit zeros
  typename G::MatrixCsr Acsrh;
  {
    std::vector<int> rpo(n + 1, 0), cio;
    std::vector<T> va;
    for (int i = 0; i < n; i++) {
      for (int p = rp[i]; p < rp[i + 1]; p++) {
        const T a = (T)v[p];
        if (a != 0) {
          cio.push_back(ci[p]);
          va.push_back(a);
        }
      }
      rpo[i + 1] = (int)cio.size();
    }
    Acsrh.resize(n, n, cio.size());
    thrust::copy(rpo.begin(), rpo.end(), Acsrh.row_offsets.begin());
    thrust::copy(cio.begin(), cio.end(), Acsrh.column_indices.begin());
    thrust::copy(va.begin(), va.end(), Acsrh.values.begin());
  }
  // 2. DB and RCM
  typename G::IntVector optReordering, optPerm, secondReorder, secondPerm, first_rows;
  typename G::IntVectorD dbRowPerm(n);
  typename G::VectorD dbRowScale, dbColScale;
  typename G::MatrixMapF scaleMap;
  G graph(false);
  const bool doRCM = maxBandwidth > 64;
  int k_db = 0;
  const int k_reorder = graph.reorder(Acsrh, false, doDB != 0, false, scale != 0, doRCM, false, optReordering, optPerm,
                                      dbRowPerm, dbRowScale, dbColScale, scaleMap, k_db);
  // 3. drop-off
  int K = k_reorder;
  T drop_actual = 0;
  if (k_reorder > maxBandwidth || dropFrac > 0) K = graph.dropOff((T)dropFrac, maxBandwidth, drop_actual);
  // 4. partitions
  int P = std::min(P_req, std::max(n / (K + 1), 1));
  bool var = varBand != 0;
  if (P == 1 || K == 0) var = false;
  // 5. variable-band assembly
  typename G::Vector WV, offDiags;
  typename G::IntVector wl, wr, permL, permR, ks_col, ks_row, ks, BOffsets;
  typename G::MatrixMap typeMap, offDiagMap, WVMap, bandedMatMap;
  typename G::MatrixCoo Acooh;
  if (var) {
    graph.assembleOffDiagMatrices(K, P, WV, offDiags, wl, wr, permL, permR, typeMap, offDiagMap, WVMap);
    graph.secondLevelReordering(K, P, secondReorder, secondPerm, first_rows);
    graph.assembleBandedMatrix(K, false, P, ks_col, ks_row, Acooh, ks, BOffsets, typeMap, bandedMatMap);
  }
  // 6. composition: combinePermutation(perm, perm2, out): out[i] = perm2[perm[i]]
  std::vector<int> oR = to_std(optReordering), oP = to_std(optPerm), db = to_std(dbRowPerm);
  std::vector<int> fR = oR, fP = oP;
  if (var) {
    std::vector<int> sR = to_std(secondReorder), sP = to_std(secondPerm);
    for (int i = 0; i < n; i++) fR[i] = oR[sR[i]];  // combinePermutation(secondReorder, optReordering)
    for (int i = 0; i < n; i++) fP[i] = sP[oP[i]];  // combinePermutation(optPerm, secondPerm)
  }
  {
    std::vector<int> t(n);
    for (int i = 0; i < n; i++) t[i] = fP[db[i]];  // combinePermutation(dbRowPerm, optPerm)
    fP.swap(t);
  }
  r.n = n;
  r.K = K;
  r.P = P;
  r.k_db = k_db;
  r.k_reorder = k_reorder;
  r.varBand = var ? 1 : 0;
  r.drop_actual = (double)drop_actual;
  r.ints[0] = db;
  r.ints[1] = oR;
  r.ints[2] = oP;
  r.ints[3] = to_std(secondReorder);
  r.ints[4] = to_std(secondPerm);
  r.ints[5] = to_std(first_rows);
  r.ints[6] = to_std(ks);
  r.ints[7] = fP;
  r.ints[8] = fR;
  r.ints[9] = to_std(wl);
  r.ints[10] = to_std(wr);
  r.ints[11] = to_std(permL);
  r.ints[12] = to_std(permR);
  r.ints[13] = to_std(ks_col);
  r.ints[14] = to_std(ks_row);
}

}  // namespace

extern "C" {

struct ref_graph_info {
  int n, K, P, k_db, k_reorder, varBand, status;
  double drop_actual;
};

// Runs the pipeline with PrecValueType float (prec_double 0) or double;
// returns a handle; its status is 0 on success, the sap::system_error
// reason on a reference exception.
void* ref_graph_run(int n, const int* rp, const int* ci, const double* v, int prec_double, int P_req, double dropFrac,
                    int doDB, int scale, int maxBandwidth, int varBand, char* msg, int msg_len) {
  RefResult* r = new RefResult();
  try {
    if (prec_double)
      run<double>(*r, n, rp, ci, v, P_req, dropFrac, doDB, scale, maxBandwidth, varBand);
    else
      run<float>(*r, n, rp, ci, v, P_req, dropFrac, doDB, scale, maxBandwidth, varBand);
  } catch (const sap::system_error& e) {
    r->status = (int)e.reason();
    r->msg = e.what();
  } catch (const thrust::system_error& e) {
    r->status = -101;
    r->msg = e.what();
  } catch (const std::exception& e) {
    r->status = -100;
    r->msg = e.what();
  }
  if (msg && msg_len > 0) {
    std::strncpy(msg, r->msg.c_str(), (size_t)msg_len - 1);
    msg[msg_len - 1] = 0;
  }
  return r;
}

void ref_graph_info_get(void* h, ref_graph_info* out) {
  const RefResult* r = (const RefResult*)h;
  out->n = r->n;
  out->K = r->K;
  out->P = r->P;
  out->k_db = r->k_db;
  out->k_reorder = r->k_reorder;
  out->varBand = r->varBand;
  out->status = r->status;
  out->drop_actual = r->drop_actual;
}

// The integer outputs, in the oracle's order (0 dbRowPerm, 1 optReordering,
// 2 optPerm, 3 secondReorder, 4 secondPerm, 5 first_rows, 6 ks, 7 finalPerm,
// 8 finalReordering, 9 offDiagWidths_left, 10 offDiagWidths_right,
// 11 offDiagPerms_left, 12 offDiagPerms_right, 13 ks_col, 14 ks_row).
long long ref_graph_ints(void* h, int which, int* out) {
  const RefResult* r = (const RefResult*)h;
  if (which < 0 || which > 14) return -1;
  const std::vector<int>& v = r->ints[which];
  if (out) std::memcpy(out, v.data(), v.size() * sizeof(int));
  return (long long)v.size();
}

void ref_graph_destroy(void* h) { delete (RefResult*)h; }

}  // extern "C"
