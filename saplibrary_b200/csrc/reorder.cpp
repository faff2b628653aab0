// Sparse reordering pipeline of the solver setup: DB maximum-product
// matching with scaling, RCM, drop-off, coupling-block assembly,
// per-partition (second-level) RCM and the variable-band layout.
//
// The graph searches are inherently sequential (Dijkstra augmenting paths,
// priority-queue BFS) and their tie order decides the permutations, which
// must equal the reference's bit for bit; they run on the host exactly as
// sap/graph.h orders them.  The data-parallel step with a transcendental,
// the DB edge weights log(rowmax / |a|), is computed on the GPU by the
// caller (the reference computes it on the device too, db.cuh:14-37), so
// the weights are the device's.
#include "reorder_pipeline.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <queue>
#include <utility>

namespace sapb {
namespace rp {

namespace {

constexpr double kInf = 1e37;  // Graph<T>::LOC_INFINITY (graph.h:287-288)

struct ByDist {  // min-heap on the tentative distance (CompareValue<double>)
  bool operator()(const std::pair<int, double>& a, const std::pair<int, double>& b) const {
    return a.second > b.second;
  }
};
struct ByDegree {  // min-heap on the degree (CompareValue<int>)
  bool operator()(const std::pair<int, int>& a, const std::pair<int, int>& b) const { return a.second > b.second; }
};

// Stable counting sort of (key, payload...) triplets into CSR order: entries
// are placed from the last to the first into decreasing slots of their key,
// which keeps their input order inside every key (graph.h:1335-1356).
template <typename V>
void csr_from_keys(int n, const std::vector<int>& key, const std::vector<int>& col, const std::vector<V>& val,
                   std::vector<int>& out_rp, std::vector<int>& out_ci, std::vector<V>& out_val) {
  const size_t m = key.size();
  out_rp.assign(n + 1, 0);
  for (size_t e = 0; e < m; e++) out_rp[key[e]]++;
  for (int i = 1; i <= n; i++) out_rp[i] += out_rp[i - 1];
  out_ci.resize(m);
  out_val.resize(m);
  for (size_t e = m; e-- > 0;) {
    int slot = --out_rp[key[e]];
    out_ci[slot] = col[e];
    out_val[slot] = val[e];
  }
  out_rp[n] = (int)m;
}

int partition_of(int r, int q, int rem) {
  int p = r / (q + 1);
  return p >= rem ? rem + (r - rem * (q + 1)) / q : p;
}

}  // namespace

// ---------------------------------------------------------------------------
// DB (graph.h:1214-1361): maximum-product matching of rows to columns by
// shortest augmenting paths, with row/column scaling from its dual values.
template <typename T>
void Pipeline<T>::db(const std::vector<double>& weight, const std::vector<double>& rowmax) {
  // weight[e] = log(rowmax[row] / |a_e|), computed on the device
  const std::vector<int>& Rp = in_rp;
  const std::vector<int>& Ci = in_ci;
  std::vector<double> u(n, 0.0), v(n, kInf);
  std::vector<int> match(n, 0), rev_match(nnz, 0);
  std::vector<char> row_done(n, 0), col_done(n, 0);
  // initial duals: u = per-row minimum weight (reduce_by_key over CSR rows)
  for (int i = 0; i < n; i++) {
    double m = 0;
    for (int e = Rp[i]; e < Rp[i + 1]; e++) m = (e == Rp[i]) ? weight[e] : std::min(m, weight[e]);
    u[i] = m;
  }
  // greedy initial matching (init_reduced_cval, graph.h:1890-1918)
  for (int i = 0; i < n; i++) {
    int best = -1;
    for (int e = Rp[i]; e < Rp[i + 1]; e++) {
      if (weight[e] > kInf / 2.0) continue;
      double red = weight[e] - u[Ci[e]];
      if (v[i] > red) { v[i] = red; best = e; }
    }
    if (best >= 0 && !row_done[Ci[best]]) {
      col_done[i] = 1;
      row_done[Ci[best]] = 1;
      match[Ci[best]] = i;
      rev_match[i] = best;
    }
  }
  for (int i = 0; i < n; i++) {
    if (!row_done[i]) u[i] = 0.0;
    if (!col_done[i]) v[i] = 0.0;
  }
  // augmenting paths (find_shortest_aug_path, graph.h:2043-2173)
  std::vector<char> inB(n, 0), visited(n, 0);
  std::vector<double> dist(n, kInf);
  std::vector<int> Bset(n, 0), irn(n, 0), prev(n, 0);
  for (int start = 0; start < n; start++) {
    if (col_done[start]) continue;
    std::priority_queue<std::pair<int, double>, std::vector<std::pair<int, double>>, ByDist> heap;
    int nb = 0;
    double lsp = 0.0, lsap = kInf;
    int cur = start, isap = -1, ksap = -1;
    prev[start] = -1;
    for (;;) {
      for (int e = Rp[cur]; e < Rp[cur + 1]; e++) {
        int r = Ci[e];
        if (inB[r] || weight[e] > kInf / 2.0) continue;
        double red = weight[e] - u[r] - v[cur];
        if (red + 1e-10 < 0) throw Error(SAP_NEGATIVE_DB_WEIGHT, "Negative reduced weight in DB.");
        double dnew = lsp + red;
        if (!(dnew < lsap)) continue;
        if (!row_done[r]) {
          lsap = dnew;
          isap = r;
          ksap = e;
          match[isap] = cur;
        } else if (dnew < dist[r]) {
          dist[r] = dnew;
          prev[match[r]] = cur;
          heap.push(std::make_pair(r, dnew));
          irn[r] = e;
        }
      }
      bool found = false;
      std::pair<int, double> top;
      while (!heap.empty()) {
        top = heap.top();
        heap.pop();
        if (!visited[top.first]) { found = true; break; }
      }
      if (!found) break;
      visited[top.first] = 1;
      lsp = top.second;
      if (lsap <= lsp) {
        visited[top.first] = 0;
        dist[top.first] = kInf;
        break;
      }
      inB[top.first] = 1;
      Bset[nb++] = top.first;
      cur = match[top.first];
    }
    if (lsap < kInf / 2.0) {
      row_done[isap] = 1;
      cur = match[isap];
      v[cur] = weight[ksap];
      while (prev[cur] >= 0) {
        match[isap] = cur;
        int nk = rev_match[cur];
        int ni = Ci[nk];
        nk = irn[ni];
        rev_match[cur] = ksap;
        cur = prev[cur];
        isap = ni;
        ksap = nk;
      }
      match[isap] = cur;
      rev_match[cur] = ksap;
      col_done[cur] = 1;
      for (int k = 0; k < nb; k++) {
        int r = Bset[k];
        int c = match[r];
        u[r] += dist[r] - lsap;
        v[c] = weight[rev_match[c]] - u[r];
        dist[r] = kInf;
        visited[r] = 0;
        inB[r] = 0;
      }
      while (!heap.empty()) {
        dist[heap.top().first] = kInf;
        heap.pop();
      }
    }
  }
  for (int i = 0; i < n; i++)
    if (!row_done[i]) throw Error(SAP_MATRIX_SINGULAR, "Singular matrix found");
  col_scale.resize(n);
  row_scale.resize(n);
  for (int i = 0; i < n; i++) col_scale[i] = std::exp(u[i]);
  for (int i = 0; i < n; i++) row_scale[i] = std::exp(v[i]) / rowmax[i];
  db_row_perm.resize(n);
  for (int c = 0; c < n; c++) db_row_perm[match[c]] = c;
  // permuted (and scaled) matrix, rows in the new order, entries stable
  std::vector<int> key(nnz), col(in_ci);
  std::vector<T> val(nnz);
  for (int i = 0; i < n; i++)
    for (int e = Rp[i]; e < Rp[i + 1]; e++) {
      key[e] = db_row_perm[i];
      val[e] = scale ? (T)(row_scale[i] * col_scale[Ci[e]]) * in_val[e] : in_val[e];
    }
  csr_from_keys(n, key, col, val, m_rp, m_ci, m_val);
}

// Symmetrised adjacency of edges [e0, e1) without self loops (duplicates
// kept), rows [nb, ne] prefix-summed, entries stable (buildTopology,
// graph.h:1764-1809).
static void symmetric_adjacency(const std::vector<int>& er, const std::vector<int>& ec, int e0, int e1, int nb,
                                int ne, int n, std::vector<int>& off, std::vector<int>& adj) {
  std::vector<int> src;
  std::vector<int> dst;
  src.reserve(2 * (size_t)(e1 - e0));
  dst.reserve(2 * (size_t)(e1 - e0));
  for (int e = e0; e < e1; e++) {
    if (er[e] == ec[e]) continue;
    src.push_back(er[e]); dst.push_back(ec[e]);
    src.push_back(ec[e]); dst.push_back(er[e]);
  }
  off.assign(n + 1, 0);
  for (int s : src) off[s]++;
  for (int i = nb + 1; i <= ne; i++) off[i] += off[i - 1];
  adj.resize(dst.size());
  for (size_t e = dst.size(); e-- > 0;) adj[--off[src[e]]] = dst[e];
}

// One BFS of the Cuthill-McKee order from `root` over nodes [nb, ne):
// children are queued in increasing `degree` order through a binary heap
// (ties broken by the heap, as in the reference), restarts take the lowest
// unvisited node.  Returns false when the queue cannot be refilled.
static bool cm_bfs(int root, int nb, int ne, int trial, const std::vector<int>& off, const std::vector<int>& adj,
                   const std::vector<int>* fixed_degree, std::vector<int>& pushed, std::vector<int>& level,
                   std::vector<int>& order, int& last_level) {
  std::queue<int> fifo;
  std::priority_queue<std::pair<int, int>, std::vector<std::pair<int, int>>, ByDegree> kids;
  level[root] = 0;
  pushed[root] = trial;
  fifo.push(root);
  int left = ne - nb, out = nb, scan = nb;
  while (left--) {
    if (fifo.empty()) {
      left++;
      int i = scan;
      while (i < ne && pushed[i] == trial) i++;
      if (i >= ne) return false;
      fifo.push(i);
      pushed[i] = trial;
      scan = i;
      continue;
    }
    int node = fifo.front();
    fifo.pop();
    order[out++] = node;
    int lv = level[node];
    for (int e = off[node]; e < off[node + 1]; e++) {
      int t = adj[e];
      if (pushed[t] == trial) continue;
      pushed[t] = trial;
      int deg = fixed_degree ? (*fixed_degree)[t] : off[t + 1] - off[t];
      kids.push(std::make_pair(t, deg));
      level[t] = lv + 1;
      last_level = lv + 1;
    }
    while (!kids.empty()) {
      fifo.push(kids.top().first);
      kids.pop();
    }
  }
  return true;
}

// RCM on the DB-reordered matrix (graph.h:1371-1584).  As in the reference:
// BFS priority is the CSR row length; the trial loop stops after the second
// trial (its level bookkeeping never advances); a later trial starts from
// the lowest-index vertex of the tracked level, picked through the degrees of
// vertices 0..count-1; the best trial's order is kept only if it lowers the
// bandwidth of the current order.
template <typename T>
int Pipeline<T>::rcm() {
  const int nz = (int)m_ci.size();
  std::vector<int> row(nz), degree(n);
  for (int i = 0; i < n; i++) {
    for (int e = m_rp[i]; e < m_rp[i + 1]; e++) row[e] = i;
    degree[i] = m_rp[i + 1] - m_rp[i];
  }
  int best_bw = 0;
  for (int e = 0; e < nz; e++) best_bw = std::max(best_bw, std::abs(row[e] - m_ci[e]));
  std::vector<int> off, adj;
  symmetric_adjacency(row, m_ci, 0, nz, 0, n, n, off, adj);
  rcm_order.resize(n);
  for (int i = 0; i < n; i++) rcm_order[i] = i;
  rcm_pos.assign(n, 0);
  std::vector<char> tried(n, 0);
  std::vector<int> pushed(n, -1), level(n, 0), order(n);
  const int tracked_level = 0;  // never advanced (graph.h:1413-1414)
  for (int trial = 0; trial < 5; trial++) {
    int root;
    if (trial == 0) {
      root = (int)(std::min_element(degree.begin(), degree.end()) - degree.begin());
    } else {
      int cnt = (int)std::count(level.begin(), level.end(), tracked_level);
      if (cnt > 1) {
        int pick = (int)(std::min_element(degree.begin(), degree.begin() + cnt) - degree.begin());
        int seen = -1;
        root = 0;
        for (int i = 0; i < n; i++)
          if (level[i] == tracked_level && ++seen == pick) { root = i; break; }
      } else {
        root = (int)(std::max_element(level.begin(), level.end()) - level.begin());
      }
      while (tried[root]) root = (root + 1) % n;
    }
    tried[root] = 1;
    int unused = 0;
    if (!cm_bfs(root, 0, n, trial, off, adj, &degree, pushed, level, order, unused)) break;
    for (int k = 0; k < n; k++) rcm_pos[order[k]] = k;
    int bw = 0;
    for (int e = 0; e < nz; e++) bw = std::max(bw, std::abs(rcm_pos[row[e]] - rcm_pos[m_ci[e]]));
    if (best_bw > bw) {
      best_bw = bw;
      rcm_order = order;
    }
    if (trial > 0) break;            // tracked level never grows: the second trial is the last
    if (best_bw <= 256) break;       // BANDWIDTH_THRESHOLD
  }
  for (int k = 0; k < n; k++) rcm_pos[rcm_order[k]] = k;
  std::vector<int> key(nz), col(nz);
  for (int e = 0; e < nz; e++) {
    key[e] = rcm_pos[row[e]];
    col[e] = rcm_pos[m_ci[e]];
  }
  std::vector<T> val = m_val;
  csr_from_keys(n, key, col, val, m_rp, m_ci, m_val);
  return best_bw;
}

// Drop-off (graph.h:598-747): bands are peeled from the outside while the
// kept sum of squares (accumulated in T, in the reference's order) stays
// >= (1 - frac) of the total.  Returns the reference's half-bandwidth, which
// is the distance of the last band peeled when any is peeled.
template <typename T>
int Pipeline<T>::drop_off(T frac, int max_bw) {
  const int nz = (int)m_ci.size();
  std::vector<int> start(n + 1, 0);
  for (int i = 0; i < n; i++)
    for (int e = m_rp[i]; e < m_rp[i + 1]; e++) start[std::abs(i - m_ci[e])]++;
  for (int d = 0, acc = 0; d < n; d++) { int c = start[d]; start[d] = acc; acc += c; }
  std::vector<int> br(nz), bc(nz);
  std::vector<T> bv(nz);
  for (int i = 0; i < n; i++)
    for (int e = m_rp[i]; e < m_rp[i + 1]; e++) {
      int s = start[std::abs(i - m_ci[e])]++;
      br[s] = i; bc[s] = m_ci[e]; bv[s] = m_val[e];
    }
  T total = T(0);
  for (int e = 0; e < nz; e++) total = total + m_val[e] * m_val[e];
  const T keep_min = (T(1) - frac) * total;
  T kept = total;
  // walk from the longest distance (the end of the bucketed list)
  auto dist_at = [&](int k) { int s = nz - 1 - k; return std::abs(br[s] - bc[s]); };
  auto sq_at = [&](int k) { int s = nz - 1 - k; return bv[s] * bv[s]; };
  int cut = 0, probe = 0, kres = dist_at(0);
  {
    int d;
    while ((d = dist_at(probe)) > max_bw) probe++;
    T s = T(0);
    for (int k = cut; k < probe; k++) s = s + sq_at(k);
    kept -= s;
    cut = probe;
    kres = d;
  }
  if (kept >= keep_min) {
    for (;;) {
      int d = dist_at(cut);
      if (d == 0) { kres = 0; break; }
      do { probe++; } while (dist_at(probe) == d);
      T band = T(0);
      for (int k = cut; k < probe; k++) band = band + sq_at(k);
      if (kept - band < keep_min) break;
      kept -= band;
      cut = probe;
      kres = d;
    }
  }
  drop_actual = T(1) - kept / total;
  const int keep = nz - cut;
  // rebuild sorted by row, then column: stable by column, then by row
  std::vector<int> cstart(n + 1, 0);
  for (int k = 0; k < keep; k++) cstart[bc[k]]++;
  for (int d = 0, acc = 0; d < n; d++) { int c = cstart[d]; cstart[d] = acc; acc += c; }
  std::vector<int> tr(keep), tc(keep);
  std::vector<T> tv(keep);
  for (int k = 0; k < keep; k++) {
    int s = cstart[bc[k]]++;
    tr[s] = br[k]; tc[s] = bc[k]; tv[s] = bv[k];
  }
  csr_from_keys(n, tr, tc, tv, m_rp, m_ci, m_val);
  return kres;
}

// Coupling blocks (assembleOffDiagMatrices, graph.h:756-898): entries inside
// a diagonal block form the diagonal matrix (CSR order kept); the others go
// to the row-major K x K coupling blocks B_i (rows of partition i, columns of
// i+1) and C_{i+1} (the converse).  Rows that couple to the next partition
// are flagged for first_rows.
template <typename T>
void Pipeline<T>::assemble_coupling(int K, int P) {
  const int q = n / P, rem = n % P;
  const size_t KK = (size_t)K * K;
  offd_size = 2 * KK * (P - 1);
  offd_idx.clear();
  offd_val.clear();
  couples_right.assign(n, 0);
  d_rp.assign(n + 1, 0);
  d_ci.clear();
  d_val.clear();
  for (int j = 0; j < n; j++) {
    const int pr = partition_of(j, q, rem);
    for (int e = m_rp[j]; e < m_rp[j + 1]; e++) {
      const int l = m_ci[e];
      const int pc = partition_of(l, q, rem);
      if (pc == pr) {
        d_ci.push_back(l);
        d_val.push_back(m_val[e]);
        d_rp[j + 1]++;
      } else if (pc > pr) {
        couples_right[j] = 1;
        const int row_end = q * pr + (pr < rem ? pr + q + 1 : rem + q);
        const int col_start = q * pc + (pc < rem ? pc : rem);
        offd_idx.push_back((long long)(pr * 2 * KK + (size_t)(j + K - row_end) * K + (l - col_start)));
        offd_val.push_back(m_val[e]);
      } else {
        const int row_start = q * pr + (pr < rem ? pr : rem);
        const int col_end = q * pc + (pc < rem ? pc + q + 1 : rem + q);
        offd_idx.push_back((long long)((pc * 2 + 1) * KK + (size_t)(j - row_start) * K + (l - col_end + K)));
        offd_val.push_back(m_val[e]);
      }
    }
  }
  for (int i = 0; i < n; i++) d_rp[i + 1] += d_rp[i];
}

// Second-level reordering (secondLevelReordering + partitionedRCM,
// graph.h:908-1008, 1593-1757): RCM inside every partition with the
// symmetrised-topology degree as BFS priority, up to 5 trials stopped by the
// level-growth rule or a bandwidth <= 128; then the diagonal matrix is
// permuted and first_rows computed.
template <typename T>
void Pipeline<T>::second_level(int K, int P) {
  const int q = n / P, rem = n % P;
  const int dz = (int)d_ci.size();
  std::vector<int> row(dz);
  for (int i = 0; i < n; i++)
    for (int e = d_rp[i]; e < d_rp[i + 1]; e++) row[e] = i;
  second_order.assign(n, 0);
  second_pos.assign(n, 0);
  std::vector<int> order(n, 0);
  std::vector<int> pnb(P + 1, 0);
  for (int p = 0; p < P; p++) pnb[p + 1] = pnb[p] + q + (p < rem ? 1 : 0);
  // One partition.  Returns false, in the parallel pass, when a trial root
  // leaves the partition (the reference's root search walks on to the next
  // index): that trial's writes reach another partition, so every partition
  // is then redone serially in order, as the reference does.
  auto part = [&](int p, bool serial) -> bool {
    const int nb = pnb[p], ne = pnb[p + 1];
    const int e0 = d_rp[nb], e1 = d_rp[ne];
    for (int i = nb; i < ne; i++) second_order[i] = i;
    int best_bw = 0;
    for (int e = e0; e < e1; e++) best_bw = std::max(best_bw, std::abs(row[e] - d_ci[e]));
    std::vector<int> off, adj;
    symmetric_adjacency(row, d_ci, e0, e1, nb, ne, n, off, adj);
    std::vector<int> rowlen(ne - nb);
    for (int i = nb; i < ne; i++) rowlen[i - nb] = d_rp[i + 1] - d_rp[i];
    std::vector<char> tried(n, 0);
    std::vector<int> pushed(n, -1), level(n, 0);
    int last_level = 0, prev_last = 0;
    for (int trial = 0; trial < 5; trial++) {
      int root;
      if (trial == 0) {
        root = (int)(std::min_element(rowlen.begin(), rowlen.end()) - rowlen.begin()) + nb;
      } else {
        int cnt = (int)std::count(level.begin() + nb, level.begin() + ne, last_level);
        if (cnt > 1) {
          int pick = (int)(std::min_element(rowlen.begin(), rowlen.begin() + cnt) - rowlen.begin());
          int seen = -1;
          root = nb;
          for (int i = nb; i < ne; i++)
            if (level[i] == last_level && ++seen == pick) { root = i; break; }
        } else {
          root = (int)(std::max_element(level.begin() + nb, level.begin() + ne) - level.begin());
        }
        while (tried[root]) root = (root + 1) % n;
      }
      if (!serial && (root < nb || root >= ne)) return false;
      tried[root] = 1;
      if (!cm_bfs(root, nb, ne, trial, off, adj, nullptr, pushed, level, order, last_level)) break;
      for (int k = nb; k < ne; k++) second_pos[order[k]] = k;
      int bw = 0;
      for (int e = e0; e < e1; e++) bw = std::max(bw, std::abs(second_pos[row[e]] - second_pos[d_ci[e]]));
      if (best_bw > bw) {
        best_bw = bw;
        std::copy(order.begin() + nb, order.begin() + ne, second_order.begin() + nb);
      }
      if (trial > 0) {
        if (prev_last >= last_level) break;
        if (1.0 * (last_level - prev_last) / prev_last < 0.01) break;
      }
      prev_last = last_level;
      if (best_bw <= 128) break;
    }
    for (int k = nb; k < ne; k++) second_pos[second_order[k]] = k;
    return true;
  };
  int ok = 1;
#pragma omp parallel for schedule(dynamic, 1) reduction(&& : ok)
  for (int p = 0; p < P; p++) ok = part(p, false) && ok;
  if (!ok) {
    second_pos.assign(n, 0);
    for (int p = 0; p < P; p++) part(p, true);
  }
  std::vector<int> key(dz), col(dz);
  for (int e = 0; e < dz; e++) {
    key[e] = second_pos[row[e]];
    col[e] = second_pos[d_ci[e]];
  }
  std::vector<T> val = d_val;
  csr_from_keys(n, key, col, val, d_rp, d_ci, d_val);
  first_rows.assign(std::max(P - 1, 0), 0);
  int last = 0;
  for (int i = 0; i < P - 1; i++) {
    last += q + (i < rem ? 1 : 0);
    first_rows[i] = last;
    for (int j = last - K; j < last; j++)
      if (couples_right[j] && first_rows[i] > second_pos[j]) first_rows[i] = second_pos[j];
  }
}

// Variable band (assembleBandedMatrix, graph.h:1093-1206): K_p is the largest
// |i - j| of the entries whose column lies in partition p.
template <typename T>
void Pipeline<T>::assemble_var_band(int P) {
  const int q = n / P, rem = n % P;
  part_k.assign(P, 0);
  for (int j = 0; j < n; j++)
    for (int e = d_rp[j]; e < d_rp[j + 1]; e++) {
      int l = d_ci[e];
      int p = partition_of(l, q, rem);
      part_k[p] = std::max(part_k[p], std::abs(l - j));
    }
}

// The whole sparse setup of transformToBandedMatrix (precond.h:1656-2101)
// up to the band layout.
template <typename T>
void Pipeline<T>::run(const std::vector<double>& weight, const std::vector<double>& rowmax) {
  stage_ms.clear();
  auto t0 = std::chrono::steady_clock::now();
  auto lap = [&](const char* name) {
    auto t1 = std::chrono::steady_clock::now();
    stage_ms.emplace_back(name, std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  };
  if (do_db) {
    db(weight, rowmax);
  } else {
    m_rp = in_rp; m_ci = in_ci; m_val = in_val;
    db_row_perm.resize(n);
    for (int i = 0; i < n; i++) db_row_perm[i] = i;
    row_scale.assign(n, 1.0);
    col_scale.assign(n, 1.0);
  }
  k_db = 0;
  for (int i = 0; i < n; i++)
    for (int e = m_rp[i]; e < m_rp[i + 1]; e++) k_db = std::max(k_db, std::abs(i - m_ci[e]));
  lap("db");
  if (max_bandwidth > 64) {
    k_reorder = rcm();
  } else {
    k_reorder = k_db;
    rcm_order.resize(n);
    rcm_pos.resize(n);
    for (int i = 0; i < n; i++) rcm_order[i] = rcm_pos[i] = i;
  }
  lap("rcm");
  if (k_reorder > max_bandwidth || drop_frac > 0) {
    K = drop_off((T)drop_frac, max_bandwidth);
  } else {
    K = k_reorder;
    drop_actual = T(0);
  }
  lap("drop_off");
  P = std::min(P_req, std::max(n / (K + 1), 1));
  if (P == 1 || K == 0) var_band = false;
  if (var_band) {
    assemble_coupling(K, P);
    lap("coupling");
    second_level(K, P);
    lap("second_level");
    assemble_var_band(P);
    lap("assemble");
  } else {
    second_order.resize(n);
    second_pos.resize(n);
    for (int i = 0; i < n; i++) second_order[i] = second_pos[i] = i;
  }
  // composed permutations (precond.h:2071-2097): band row of input row i,
  // and input column of band column k
  final_pos.resize(n);
  final_order.resize(n);
  for (int k = 0; k < n; k++) final_order[k] = rcm_order[second_order[k]];
  for (int i = 0; i < n; i++) final_pos[i] = second_pos[rcm_pos[db_row_perm[i]]];
  lap("compose");
}

template class Pipeline<float>;
template class Pipeline<double>;

}  // namespace rp
}  // namespace sapb
