// Host reordering pipeline of the sparse setup (see reorder.cpp).
#pragma once

#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/sap_b200.h"

namespace sapb {

#ifndef SAPB_ERROR_DEFINED
#define SAPB_ERROR_DEFINED
struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
#endif

namespace rp {

// a[i + 1] += a[i] for i = 0 .. n-1 (running sums of a[1..n] after a[0]),
// in parallel blocks above a size threshold; integer sums, so the result
// equals the serial loop's.
void prefix_sum(int* a, int n);

// T is the preconditioner value type: the reference runs the whole
// reordering on the matrix converted to it (precond.h:1667-1713).
template <typename T>
class Pipeline {
 public:
  // input: CSR in T with explicit zeros removed
  int n = 0, nnz = 0;
  std::vector<int> in_rp, in_ci;
  std::vector<T> in_val;
  // options
  bool do_db = true, scale = true, var_band = true;
  double drop_frac = 0;
  int max_bandwidth = std::numeric_limits<int>::max();
  int P_req = 1;

  // outputs
  std::vector<int> db_row_perm;                  // input row i -> row db_row_perm[i]
  std::vector<double> row_scale, col_scale;      // DB scalings (double)
  std::vector<int> rcm_order, rcm_pos;           // RCM: position -> node, node -> position
  std::vector<int> second_order, second_pos;     // second level, same convention
  std::vector<int> final_pos, final_order;       // composed: input row -> band row; band col -> input col
  std::vector<int> first_rows;
  // coupling blocks (row-major K x K, B_t at 2t, C_t at 2t+1) as entries of
  // the dense [P-1][2][K][K] layout: index and value
  std::vector<long long> offd_idx;
  std::vector<T> offd_val;
  size_t offd_size = 0;
  std::vector<int> part_k;                       // K_p of the variable band
  int k_db = 0, k_reorder = 0, K = 0, P = 1;
  T drop_actual = T(0);

  // working matrices: the reordered matrix and its diagonal blocks (CSR in T)
  std::vector<int> m_rp, m_ci, d_rp, d_ci;
  std::vector<T> m_val, d_val;
  std::vector<char> couples_right;

  // scratch kept across runs of the same object (a repeated setup reuses
  // its memory instead of allocating and page-faulting it again)
  std::vector<int> ws_i0, ws_i1, ws_i2, ws_off, ws_adj, ws_cnt, tmp_rp, tmp_ci;
  std::vector<T> ws_t0, tmp_val;
  // per-node state of the DB search and of the BFS trials (refilled in
  // parallel by every run)
  std::vector<double> db_u, db_v, db_dist;
  std::vector<int> db_match, db_bset, db_irn, db_prev, db_owner;
  std::vector<char> db_rowdone, db_coldone, db_inb, db_visited;
  std::vector<char> bfs_tried;
  std::vector<int> bfs_pushed, bfs_level, bfs_order, bfs_claim, bfs_degree;
  // per partition of the second level: its adjacency, row lengths and BFS
  // queue (kept, so that the partitions' threads do not allocate and fault
  // in new pages side by side on every setup)
  struct PartScratch {
    std::vector<int> off, adj, pos, rowlen, fifo;
  };
  std::vector<PartScratch> part_scratch;

  // wall time of the stages of run(), in order (ms)
  std::vector<std::pair<const char*, double>> stage_ms;
  double stage(const char* name) const {
    double t = 0;
    for (const auto& s : stage_ms)
      if (std::string(s.first) == name) t += s.second;
    return t;
  }

  // weight[e] = log(rowmax[row(e)] / |a_e|) and rowmax, both from the device
  void run(const double* weight, const double* rowmax);

 private:
  void db(const double* weight, const double* rowmax);
  int rcm();
  int drop_off(T frac, int max_bw);
  void assemble_coupling(int K, int P);
  void second_level(int K, int P);
  void assemble_var_band(int P);
};

}  // namespace rp
}  // namespace sapb
