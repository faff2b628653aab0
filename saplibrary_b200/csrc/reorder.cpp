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
#include <climits>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <queue>
#include <thread>
#include <type_traits>
#include <utility>

#include <omp.h>

namespace sapb {
namespace rp {

void prefix_sum(int* a, int n) {
  const int nt = std::max(1, std::min(omp_get_max_threads(), 16));
  if (nt == 1 || n < (1 << 16)) {
    for (int i = 0; i < n; i++) a[i + 1] += a[i];
    return;
  }
  std::vector<int> part(nt + 1, 0);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num(), nth = omp_get_num_threads();
    const int i0 = (int)((long long)n * t / nth), i1 = (int)((long long)n * (t + 1) / nth);
    int s = 0;
    for (int i = i0; i < i1; i++) s += a[i + 1];
    part[t + 1] = s;
#pragma omp barrier
    int run = a[0];
    for (int u = 0; u < t; u++) run += part[u + 1];
    for (int i = i0; i < i1; i++) {
      run += a[i + 1];
      a[i + 1] = run;
    }
  }
}

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

// Rows moved as whole units: row oldrow[k] of (rp, ci, val) becomes row k
// with its entries in their order and columns relabelled through colmap
// (none when null).  This is exactly what the stable counting sort by
// key = new position of the row (csr_from_keys) produces, built in parallel
// over the new rows (the writes stream; a band-like result keeps the reads
// through colmap and value_of near each other).
// value_of(r, e) gives the value written for entry e of old row r.
template <typename V, typename F>
void permute_rows_with(int n, const std::vector<int>& rp, const std::vector<int>& ci, F value_of,
                       const int* oldrow, const std::vector<int>* colmap, std::vector<int>& out_rp,
                       std::vector<int>& out_ci, std::vector<V>& out_val) {
  out_rp.resize(n + 1);
  out_rp[0] = 0;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; k++) out_rp[k + 1] = rp[oldrow[k] + 1] - rp[oldrow[k]];
  prefix_sum(out_rp.data(), n);
  out_ci.resize(ci.size());
  out_val.resize(ci.size());
  const int* cm = colmap ? colmap->data() : nullptr;
#pragma omp parallel for schedule(static, 4096)
  for (int k = 0; k < n; k++) {
    const int r = oldrow[k];
    int d = out_rp[k];
    for (int e = rp[r]; e < rp[r + 1]; e++, d++) {
      out_ci[d] = cm ? cm[ci[e]] : ci[e];
      out_val[d] = value_of(r, e);
    }
  }
}

template <typename V>
void permute_rows(int n, const std::vector<int>& rp, const std::vector<int>& ci, const std::vector<V>& val,
                  const std::vector<int>& oldrow, const std::vector<int>* colmap, std::vector<int>& out_rp,
                  std::vector<int>& out_ci, std::vector<V>& out_val) {
  const V* v = val.data();
  permute_rows_with(n, rp, ci, [v](int, int e) { return v[e]; }, oldrow.data(), colmap, out_rp, out_ci, out_val);
}

int partition_of(int r, int q, int rem) {
  int p = r / (q + 1);
  return p >= rem ? rem + (r - rem * (q + 1)) / q : p;
}

}  // namespace

// v resized to n (its memory kept across runs) with every element set to x,
// in parallel
template <typename V, typename X>
V& pfill(V& v, size_t n, X x) {
  if (v.size() != n) v.resize(n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n; i++) v[i] = x;
  return v;
}

// ---------------------------------------------------------------------------
// DB (graph.h:1214-1361): maximum-product matching of rows to columns by
// shortest augmenting paths, with row/column scaling from its dual values.
template <typename T>
void Pipeline<T>::db(const double* weight, const double* rowmax) {
  // weight[e] = log(rowmax[row] / |a_e|), computed on the device
  const std::vector<int>& Rp = in_rp;
  const std::vector<int>& Ci = in_ci;
  std::vector<double>& u = pfill(db_u, n, 0.0);
  std::vector<double>& v = pfill(db_v, n, kInf);
  std::vector<int>& match = pfill(db_match, n, 0);
  std::vector<int>& rev_match = pfill(ws_i0, n, 0);  // per column: its matched entry
  std::vector<char>& row_done = pfill(db_rowdone, n, (char)0);
  std::vector<char>& col_done = pfill(db_coldone, n, (char)0);
  // initial duals: u = per-row minimum weight (reduce_by_key over CSR rows)
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    double m = 0;
    for (int e = Rp[i]; e < Rp[i + 1]; e++) m = (e == Rp[i]) ? weight[e] : std::min(m, weight[e]);
    u[i] = m;
  }
  // greedy initial matching (init_reduced_cval, graph.h:1890-1918): every
  // column's smallest reduced weight and its entry are independent of the
  // others (parallel); the claims, made in column order there, give each
  // row to the lowest column whose best entry lies in it, which is what the
  // parallel minimum over those columns (owner) gives
  std::vector<int>& best_e = ws_i1;
  std::vector<int>& best_r = ws_i2;
  std::vector<int>& owner = pfill(db_owner, n, INT_MAX);
  best_e.resize(n);
  best_r.resize(n);
  // every row holds its largest entry at weight log(1) = +0, so the row
  // minima u are +0 as a rule, and weight - (+0) is weight bit for bit: the
  // scattered reads of u are then skipped
  bool u_zero = true;
#pragma omp parallel for schedule(static) reduction(&& : u_zero)
  for (int i = 0; i < n; i++) u_zero = u_zero && u[i] == 0.0 && !std::signbit(u[i]);
  auto column_best = [&](auto skip_u) {
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; i++) {
      int best = -1;
      double vi = kInf;
      for (int e = Rp[i]; e < Rp[i + 1]; e++) {
        if (weight[e] > kInf / 2.0) continue;
        const double red = decltype(skip_u)::value ? weight[e] : weight[e] - u[Ci[e]];
        if (vi > red) { vi = red; best = e; }
      }
      v[i] = vi;
      best_e[i] = best;
      best_r[i] = best >= 0 ? Ci[best] : -1;
    }
  };
  if (u_zero) column_best(std::true_type{});
  else column_best(std::false_type{});
  int* own = owner.data();
  // a first pass of plain stores leaves in owner[r] one of the columns that
  // chose r (writes to different rows overlap; atomic updates would not);
  // the second lowers it to the smallest, atomically, where it is not
  // already (only rows chosen by several columns)
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    const int r = best_r[i];
    if (r >= 0 && i < __atomic_load_n(own + r, __ATOMIC_RELAXED)) __atomic_store_n(own + r, i, __ATOMIC_RELAXED);
  }
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    const int r = best_r[i];
    if (r < 0) continue;
    int cur = __atomic_load_n(own + r, __ATOMIC_RELAXED);
    while (i < cur && !__atomic_compare_exchange_n(own + r, &cur, i, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
  }
  // the claims written on each side in index order (scattered byte writes
  // from many threads would share cache lines)
#pragma omp parallel for schedule(static, 4096)
  for (int r = 0; r < n; r++) {
    if (own[r] == INT_MAX) continue;
    row_done[r] = 1;
    match[r] = own[r];
  }
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    const int r = best_r[i];
    if (r >= 0 && own[r] == i) {
      col_done[i] = 1;
      rev_match[i] = best_e[i];
    }
  }
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    if (!row_done[i]) u[i] = 0.0;
    if (!col_done[i]) v[i] = 0.0;
  }
  // augmenting paths (find_shortest_aug_path, graph.h:2043-2173)
  std::vector<char>& inB = pfill(db_inb, n, (char)0);
  std::vector<char>& visited = pfill(db_visited, n, (char)0);
  std::vector<double>& dist = pfill(db_dist, n, kInf);
  std::vector<int>& Bset = pfill(db_bset, n, 0);
  std::vector<int>& irn = pfill(db_irn, n, 0);
  std::vector<int>& prev = pfill(db_prev, n, 0);
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
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    col_scale[i] = std::exp(u[i]);
    row_scale[i] = std::exp(v[i]) / rowmax[i];
  }
  db_row_perm.resize(n);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < n; c++) db_row_perm[match[c]] = c;
  // permuted (and scaled) matrix, rows in the new order, entries stable
  const double* rs = row_scale.data();
  const double* cs = col_scale.data();
  const int* cip = Ci.data();
  const T* a = in_val.data();
  const bool sc = scale;
  // (row match[c] moves to position c)
  permute_rows_with(
      n, Rp, Ci, [=](int i, int e) { return sc ? (T)(rs[i] * cs[cip[e]]) * a[e] : a[e]; }, match.data(), nullptr,
      m_rp, m_ci, m_val);
}

// Symmetrised adjacency of edges [e0, e1) without self loops (duplicates
// kept), rows [nb, ne] prefix-summed, entries stable (buildTopology,
// graph.h:1764-1809).
// obase: node x's range is off[x - obase]; 0 gives an array of n + 1 over
// all nodes, nb one of ne - nb + 1 over the partition's nodes only.
static void symmetric_adjacency(const std::vector<int>& rp, const std::vector<int>& ci, int nb, int ne, int n,
                                std::vector<int>& off, std::vector<int>& adj, int obase, std::vector<int>& pos) {
  // the edges are the entries of rows [nb, ne) in CSR order; each edge
  // (r, c), r != c, contributes (r -> c) then (c -> r); a node's neighbours
  // keep the order of these contributions
  off.assign(obase ? ne - nb + 1 : n + 1, 0);
  auto o = [&](int x) -> int& { return off[x - obase]; };  // x in [nb, ne]
  for (int r = nb; r < ne; r++)
    for (int e = rp[r]; e < rp[r + 1]; e++) {
      if (ci[e] == r) continue;
      o(r)++;
      o(ci[e])++;
    }
  for (int i = nb + 1; i <= ne; i++) o(i) += o(i - 1);
  for (int i = ne - 1; i >= nb; i--) o(i) = i > nb ? o(i - 1) : 0;  // exclusive starts
  adj.resize(o(ne));
  pos.assign(off.begin() + (nb - obase), off.begin() + (ne - obase));
  for (int r = nb; r < ne; r++)
    for (int e = rp[r]; e < rp[r + 1]; e++) {
      const int c = ci[e];
      if (r == c) continue;
      adj[pos[r - nb]++] = c;
      adj[pos[c - nb]++] = r;
    }
}

// The same adjacency for a whole CSR matrix (rows rp, columns ci), built in
// parallel.  Node x's list in the serial builder's order is: the rows r < x
// of the entries (r, x) in entry order, then row x's own columns, then the
// rows r > x of the entries (r, x).  The column lists are a stable transpose:
// every thread counts the columns of its block of rows (counters only over
// the column range its rows reach), the counts are turned into
// per-(column, thread) offsets, and each thread places its rows in order,
// so every column lists its rows in entry order without sorting.
static void symmetric_adjacency_csr(int n, const std::vector<int>& rp, const std::vector<int>& ci,
                                    std::vector<int>& off, std::vector<int>& adj, std::vector<int>& cnt,
                                    std::vector<int>& cstart, std::vector<int>& tr) {
  const int nt = std::max(1, std::min(omp_get_max_threads(), 16));
  cstart.resize(n + 1);
  off.resize(n + 1);
  off[0] = 0;
  cstart[0] = 0;
  // per thread: the column range [lo, hi] its rows reach (a band matrix
  // keeps it near the thread's rows), where its counters live
  std::vector<int> lo(nt, INT_MAX), hi(nt, -1), sa(nt + 1, 0), sb(nt + 1, 0);
  std::vector<size_t> base(nt + 1, 0);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num(), nth = omp_get_num_threads();
    const int r0 = (int)((long long)n * t / nth), r1 = (int)((long long)n * (t + 1) / nth);
    int l = INT_MAX, h = -1;
    for (int r = r0; r < r1; r++) {
      int own = 0;
      for (int e = rp[r]; e < rp[r + 1]; e++) {
        const int x = ci[e];
        if (x != r) {
          own++;
          l = std::min(l, x);
          h = std::max(h, x);
        }
      }
      off[r + 1] = own;
    }
    lo[t] = l;
    hi[t] = h;
#pragma omp barrier
#pragma omp single
    {
      for (int u = 0; u < nth; u++) base[u + 1] = base[u] + (size_t)std::max(0, hi[u] - lo[u] + 1);
      cnt.resize(base[nth]);
    }
    int* c = cnt.data() + base[t];  // counter of column x at c[x - l]
    std::fill(c, c + std::max(0, h - l + 1), 0);
    for (int r = r0; r < r1; r++)
      for (int e = rp[r]; e < rp[r + 1]; e++)
        if (ci[e] != r) c[ci[e] - l]++;
#pragma omp barrier
    // per column: the threads' counts turned into their offsets inside the
    // column, the column's total in cstart[x + 1]
#pragma omp for schedule(static)
    for (int x = 0; x < n; x++) {
      int sum = 0;
      for (int u = 0; u < nth; u++) {
        if (x < lo[u] || x > hi[u]) continue;
        int& v = cnt[base[u] + (x - lo[u])];
        const int k = v;
        v = sum;
        sum += k;
      }
      cstart[x + 1] = sum;
    }
    // prefix sums (parallel, in two passes): cstart over the column totals,
    // off over own + column counts
    const int x0 = (int)((long long)n * t / nth), x1 = (int)((long long)n * (t + 1) / nth);
    {
      int s1 = 0, s2 = 0;
      for (int i = x0; i < x1; i++) {
        s1 += off[i + 1] + cstart[i + 1];
        s2 += cstart[i + 1];
      }
      sa[t + 1] = s1;
      sb[t + 1] = s2;
    }
#pragma omp barrier
    {
      int s1 = 0, s2 = 0;
      for (int u = 0; u < t; u++) {
        s1 += sa[u + 1];
        s2 += sb[u + 1];
      }
      for (int i = x0; i < x1; i++) {
        s1 += off[i + 1] + cstart[i + 1];
        s2 += cstart[i + 1];
        off[i + 1] = s1;
        cstart[i + 1] = s2;
      }
    }
#pragma omp barrier
#pragma omp single
    {
      tr.resize(cstart[n]);
      adj.resize(off[n]);
    }
    for (int r = r0; r < r1; r++)
      for (int e = rp[r]; e < rp[r + 1]; e++) {
        const int x = ci[e];
        if (x != r) tr[cstart[x] + c[x - l]++] = r;
      }
#pragma omp barrier
#pragma omp for schedule(static)
    for (int x = 0; x < n; x++) {
      int w = off[x], k = cstart[x];
      const int k1 = cstart[x + 1];
      for (; k < k1 && tr[k] < x; k++) adj[w++] = tr[k];
      for (int e = rp[x]; e < rp[x + 1]; e++)
        if (ci[e] != x) adj[w++] = ci[e];
      for (; k < k1; k++) adj[w++] = tr[k];
    }
  }
}

// One BFS of the Cuthill-McKee order from `root` over nodes [nb, ne):
// children are queued in increasing `degree` order through a binary heap
// (ties broken by the heap, as in the reference), restarts take the lowest
// unvisited node.  Returns false when the queue cannot be refilled.
// The order's bandwidth is the largest distance from a queued node to the
// node that queued it (see cm_bfs_levels).  With give_up > 0 the order is
// given up (*gave_up set) once that distance reaches give_up, and the rest
// of the search only fills level[] and last_level, queueing children in
// adjacency order: the levels and the last level do not depend on the
// order inside a batch.
static bool cm_bfs(int root, int nb, int ne, int trial, const std::vector<int>& offv, const std::vector<int>& adj,
                   const std::vector<int>* fixed_degree, std::vector<int>& pushed, std::vector<int>& level,
                   std::vector<int>& order, int& last_level, int obase, std::vector<int>& fifo, int give_up = 0,
                   bool* gave_up = nullptr) {
  auto off = [&](int x) { return offv[x - obase]; };  // node x's range starts at off(x) (see symmetric_adjacency)
  // FIFO as an array: every node enters at most once per trial
  if (fifo.size() < (size_t)(ne - nb) + 2) fifo.resize((size_t)(ne - nb) + 2);
  size_t head = 0, tail = 0;
  std::priority_queue<std::pair<int, int>, std::vector<std::pair<int, int>>, ByDegree> kids;
  level[root] = 0;
  pushed[root] = trial;
  fifo[tail++] = root;
  int left = ne - nb, out = nb, scan = nb;
  bool ordered = true;
  long long bw = 0;
  if (gave_up) *gave_up = false;
  while (left--) {
    if (head == tail) {
      left++;
      int i = scan;
      while (i < ne && pushed[i] == trial) i++;
      if (i >= ne) return false;
      fifo[tail++] = i;
      pushed[i] = trial;
      scan = i;
      continue;
    }
    int node = fifo[head++];
    order[out++] = node;
    int lv = level[node];
    if (!ordered) {
      for (int e = off(node); e < off(node + 1); e++) {
        int t = adj[e];
        if (pushed[t] == trial) continue;
        pushed[t] = trial;
        fifo[tail++] = t;
        level[t] = lv + 1;
        last_level = lv + 1;
      }
      continue;
    }
    for (int e = off(node); e < off(node + 1); e++) {
      int t = adj[e];
      if (pushed[t] == trial) continue;
      pushed[t] = trial;
      int deg = fixed_degree ? (*fixed_degree)[t] : off(t + 1) - off(t);
      kids.push(std::make_pair(t, deg));
      level[t] = lv + 1;
      last_level = lv + 1;
    }
    if (!kids.empty()) bw = std::max(bw, (long long)(tail + kids.size() - 1) - (long long)(head - 1));
    while (!kids.empty()) {
      fifo[tail++] = kids.top().first;
      kids.pop();
    }
    if (give_up > 0 && bw >= give_up) {
      ordered = false;
      if (gave_up) *gave_up = true;
    }
  }
  return true;
}

// cm_bfs over the whole graph (nodes [0, n), degrees fixed), level by
// level and in parallel, with the same result.  The FIFO is consumed in
// batches: a batch is everything queued while the previous batch was
// scanned.  A node queued from a batch belongs to the first node of the
// batch, in FIFO order, that meets it unqueued (smallest claim), and every
// claimer queues its nodes through the same degree heap in its adjacency
// order, so the concatenation equals the serial queue.  Every thread owns a
// contiguous range of the batch: one scan of its nodes' adjacency lowers the
// claims and records, per node, the neighbours it claimed at that moment;
// after a barrier each node keeps those it still holds (in adjacency order)
// and queues them through the heap into the thread's buffer, and the
// buffers, concatenated in thread order, are the next batch.  Small batches
// are scanned serially.  claim[] is INT_MAX everywhere on entry and on
// return.
// A queued node's neighbours placed before it are its claimer and nodes
// after the claimer (an earlier neighbour would have queued it sooner), so
// the order's bandwidth is the largest distance from a node to its claimer.
// With give_up > 0 the order is given up (*gave_up set) once that distance
// reaches give_up: it cannot have a bandwidth below it.  The search then
// stops (returns false), or, with keep_levels, goes on without ordering to
// fill level[]: a node's level is its batch's, and the batches hold the same
// nodes (the unqueued neighbours of the previous batch, or a restart) in
// whatever order they are queued, so the levels equal the ordered search's.
static bool cm_bfs_levels(int root, int n, int trial, const std::vector<int>& off, const std::vector<int>& adj,
                          const std::vector<int>& degree, std::vector<int>& pushed, std::vector<int>& level,
                          std::vector<int>& order, std::vector<int>& claim, int give_up = 0,
                          bool* gave_up = nullptr, bool keep_levels = false) {
  constexpr int kSerialBatch = 384;
  const int nt = std::max(1, std::min(omp_get_max_threads(), 16));
  int h0 = 0, t0 = 1, scan = 0, serial_total = 0;
  bool ok = true;
  level[root] = 0;
  pushed[root] = trial;
  order[0] = root;
  int* cl = claim.data();
  std::vector<int> made(nt + 1, 0);  // nodes queued by each thread in this batch
  std::vector<int> reach(nt, 0);     // per thread: largest position - claimer position in this batch
  int bw = 0;
  bool unordered = false;  // the order was given up: levels only
  if (gave_up) *gave_up = false;
  using Kids = std::priority_queue<std::pair<int, int>, std::vector<std::pair<int, int>>, ByDegree>;
#pragma omp parallel num_threads(nt)
  {
    Kids kids;
    const int tid = omp_get_thread_num(), nth = omp_get_num_threads();
    std::vector<int> cand, per_node, out;  // claimed neighbours, their count per node, queued nodes
    for (;;) {
      const int m = t0 - h0, next = t0;  // shared, stable until the closing single
      if (m == 0) break;
      const bool serial = m < kSerialBatch, unord = unordered;
      if (unord) {
        // levels only: every thread queues the unqueued neighbours of its
        // range of the batch, each taken once by whichever thread marks it
        const int k0 = h0 + (int)((long long)m * tid / nth), k1 = h0 + (int)((long long)m * (tid + 1) / nth);
        out.clear();
        int* pu = pushed.data();
        for (int k = k0; k < k1; k++) {
          const int u = order[k], lv = level[u] + 1;
          for (int e = off[u]; e < off[u + 1]; e++) {
            const int t = adj[e];
            int cur = __atomic_load_n(pu + t, __ATOMIC_RELAXED);
            if (cur == trial) continue;
            if (__atomic_compare_exchange_n(pu + t, &cur, trial, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
              level[t] = lv;
              out.push_back(t);
            }
          }
        }
        made[tid + 1] = (int)out.size();
#pragma omp barrier
        int start = next;
        for (int u = 1; u <= tid; u++) start += made[u];
        std::copy(out.begin(), out.end(), order.begin() + start);
      } else if (serial) {
#pragma omp single
        {
          int tail = t0;
          for (int k = h0; k < t0; k++) {
            const int u = order[k], lv = level[u];
            for (int e = off[u]; e < off[u + 1]; e++) {
              const int t = adj[e];
              if (pushed[t] == trial) continue;
              pushed[t] = trial;
              kids.push(std::make_pair(t, degree[t]));
              level[t] = lv + 1;
            }
            if (!kids.empty()) bw = std::max(bw, tail + (int)kids.size() - 1 - k);
            while (!kids.empty()) {
              order[tail++] = kids.top().first;
              kids.pop();
            }
          }
          serial_total = tail - t0;
        }
      } else {
        const int k0 = h0 + (int)((long long)m * tid / nth), k1 = h0 + (int)((long long)m * (tid + 1) / nth);
        cand.clear();
        per_node.resize(k1 - k0);
        for (int k = k0; k < k1; k++) {
          const int u = order[k];
          const size_t c0 = cand.size();
          for (int e = off[u]; e < off[u + 1]; e++) {
            const int t = adj[e];
            if (pushed[t] == trial) continue;
            int cur = __atomic_load_n(cl + t, __ATOMIC_RELAXED);
            while (k < cur) {
              if (__atomic_compare_exchange_n(cl + t, &cur, k, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
                cand.push_back(t);
                break;
              }
            }
          }
          per_node[k - k0] = (int)(cand.size() - c0);
        }
#pragma omp barrier
        // a neighbour is kept by the node whose claim survived (one node of
        // one thread holds it); the others see another claim or INT_MAX
        out.clear();
        size_t c = 0;
        int far = INT_MIN;  // largest (index in out) - claimer position
        for (int k = k0; k < k1; k++) {
          const int lv = level[order[k]] + 1;
          for (const size_t c1 = c + per_node[k - k0]; c < c1; c++) {
            const int t = cand[c];
            if (__atomic_load_n(cl + t, __ATOMIC_RELAXED) != k) continue;
            __atomic_store_n(cl + t, INT_MAX, __ATOMIC_RELAXED);
            pushed[t] = trial;
            level[t] = lv;
            kids.push(std::make_pair(t, degree[t]));
          }
          if (!kids.empty()) far = std::max(far, (int)(out.size() + kids.size()) - 1 - k);
          while (!kids.empty()) {
            out.push_back(kids.top().first);
            kids.pop();
          }
        }
        made[tid + 1] = (int)out.size();
#pragma omp barrier
        int start = next;  // (t0 may already be advanced by the closing single)
        for (int u = 1; u <= tid; u++) start += made[u];
        reach[tid] = far == INT_MIN ? 0 : start + far;
        std::copy(out.begin(), out.end(), order.begin() + start);
      }
#pragma omp single
      {
        int total = serial_total;
        if (unord || !serial) {
          total = 0;
          for (int u = 1; u <= nth; u++) {
            total += made[u];
            if (!unord) bw = std::max(bw, reach[u - 1]);
          }
        }
        h0 = t0;
        t0 += total;
        bool stop = false;
        if (!unord && give_up > 0 && bw >= give_up) {
          if (gave_up) *gave_up = true;
          if (keep_levels) {
            unordered = true;
          } else {
            ok = false;
            stop = true;
            h0 = t0;
          }
        }
        if (!stop && t0 == h0 && t0 < n) {  // queue empty: restart at the lowest unqueued node
          int i = scan;
          while (i < n && pushed[i] == trial) i++;
          if (i >= n) {
            ok = false;
          } else {
            order[t0++] = i;
            pushed[i] = trial;
            scan = i;
          }
        }
        if (t0 == n) h0 = t0;  // every node queued: the rest adds nothing
      }
    }
  }
  return ok;
}

// RCM on the DB-reordered matrix (graph.h:1371-1584).  As in the reference:
// BFS priority is the CSR row length; the trial loop stops after the second
// trial (its level bookkeeping never advances); a later trial starts from
// the lowest-index vertex of the tracked level, picked through the degrees of
// vertices 0..count-1; the best trial's order is kept only if it lowers the
// bandwidth of the current order.
template <typename T>
int Pipeline<T>::rcm() {
  std::vector<int>& degree = bfs_degree;
  degree.resize(n);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) degree[i] = m_rp[i + 1] - m_rp[i];
  int best_bw = k_db;  // the current order's bandwidth (same matrix)
  std::vector<int>& off = ws_off;
  std::vector<int>& adj = ws_adj;
  symmetric_adjacency_csr(n, m_rp, m_ci, off, adj, ws_cnt, ws_i1, ws_i2);
  rcm_order.resize(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) rcm_order[i] = i;
  pfill(rcm_pos, n, 0);
  std::vector<char>& tried = pfill(bfs_tried, n, (char)0);
  std::vector<int>& pushed = pfill(bfs_pushed, n, -1);
  std::vector<int>& level = pfill(bfs_level, n, 0);
  std::vector<int>& order = pfill(bfs_order, n, 0);
  std::vector<int>& claim = pfill(bfs_claim, n, INT_MAX);
  const int tracked_level = 0;  // never advanced (graph.h:1413-1414)
  bool kept = false;
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
    // a trial's order only matters if it lowers the bandwidth: the search
    // gives it up as soon as it cannot; the first trial still fills its
    // levels (the next trial's root comes from them), the last one stops
    bool gave_up = false;
    if (!cm_bfs_levels(root, n, trial, off, adj, degree, pushed, level, order, claim, best_bw, &gave_up,
                       trial == 0))
      break;
    if (!gave_up) {
#pragma omp parallel for schedule(static)
      for (int k = 0; k < n; k++) rcm_pos[order[k]] = k;
      int bw = 0;
#pragma omp parallel for reduction(max : bw) schedule(static, 4096)
      for (int i = 0; i < n; i++) {
        const int pi = rcm_pos[i];
        for (int e = m_rp[i]; e < m_rp[i + 1]; e++) bw = std::max(bw, std::abs(pi - rcm_pos[m_ci[e]]));
      }
      if (best_bw > bw) {
        best_bw = bw;
        rcm_order = order;
        kept = true;
      }
    }
    if (trial > 0) break;            // tracked level never grows: the second trial is the last
    if (best_bw <= 256) break;       // BANDWIDTH_THRESHOLD
  }
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; k++) rcm_pos[rcm_order[k]] = k;
  // no trial lowered the bandwidth: the order is the identity and the
  // permuted matrix would equal the current one entry for entry
  if (!kept) return best_bw;
  tmp_rp.swap(m_rp);
  tmp_ci.swap(m_ci);
  tmp_val.swap(m_val);
  permute_rows(n, tmp_rp, tmp_ci, tmp_val, rcm_order, &rcm_pos, m_rp, m_ci, m_val);
  return best_bw;
}

// Drop-off (graph.h:598-747): bands are peeled from the outside while the
// kept sum of squares (accumulated in T, in the reference's order) stays
// >= (1 - frac) of the total.  Returns the reference's half-bandwidth, which
// is the distance of the last band peeled when any is peeled.
template <typename T>
int Pipeline<T>::drop_off(T frac, int max_bw) {
  const int nz = (int)m_ci.size();
  // The reference's bucketed list: entries ordered by distance |i - j|, rows
  // ascending and CSR order inside a distance group.  Group d occupies
  // [gstart[d], gstart[d+1]); only the values are needed (for the squares),
  // and only of the groups the walk below reaches.  Built in parallel as a
  // stable bucket sort: every thread counts the distances of its block of
  // rows (and sums their squares in double), the counts become
  // per-(distance, block) offsets, and each block's values are placed in
  // order.  Values are placed for the groups down to a few below where the
  // same walk over the double sums stops; the exact walk fills the rest
  // first if it goes further.
  // The sum of squares of all entries is a sequential sum in entry order
  // (the reference's order): one extra thread runs it meanwhile.
  T total = T(0);
  std::thread squares([&] {
    T s = T(0);
    for (int e = 0; e < nz; e++) s = s + m_val[e] * m_val[e];
    total = s;
  });
  // the passes beside it leave that thread a core
  const int nb = std::max(1, std::min(omp_get_max_threads() - 1, 16));  // threads and row blocks
  int dmax = 0;
#pragma omp parallel for schedule(static, 4096) reduction(max : dmax) num_threads(nb)
  for (int i = 0; i < n; i++)
    for (int e = m_rp[i]; e < m_rp[i + 1]; e++) dmax = std::max(dmax, std::abs(i - m_ci[e]));
  const int nd = dmax + 1;
  std::vector<int>& gstart = ws_i1;
  gstart.resize(nd + 1);
  std::vector<T>& bv = ws_t0;
  bv.resize(nz);
  std::vector<int>& cnt = ws_cnt;
  cnt.resize((size_t)nb * nd);
  std::vector<double> sq((size_t)nb * nd);
  auto block = [&](int u) { return (int)((long long)n * u / nb); };
#pragma omp parallel for schedule(static, 1) num_threads(nb)
  for (int u = 0; u < nb; u++) {
    int* c = cnt.data() + (size_t)u * nd;
    double* q = sq.data() + (size_t)u * nd;
    std::fill(c, c + nd, 0);
    std::fill(q, q + nd, 0.0);
    for (int i = block(u); i < block(u + 1); i++)
      for (int e = m_rp[i]; e < m_rp[i + 1]; e++) {
        const int d = std::abs(i - m_ci[e]);
        c[d]++;
        q[d] += (double)m_val[e] * (double)m_val[e];
      }
  }
  std::vector<double> gsq(nd, 0.0);
  {
    int run = 0;
    for (int d = 0; d < nd; d++) {
      gstart[d] = run;
      for (int u = 0; u < nb; u++) {
        int& v = cnt[(size_t)u * nd + d];
        const int k = v;
        v = run;
        run += k;
        gsq[d] += sq[(size_t)u * nd + d];
      }
    }
    gstart[nd] = run;
  }
  // place the values of groups [lo, hi)
  auto place = [&](int lo, int hi) {
#pragma omp parallel for schedule(static, 1) num_threads(nb)
    for (int u = 0; u < nb; u++) {
      int* c = cnt.data() + (size_t)u * nd;
      for (int i = block(u); i < block(u + 1); i++)
        for (int e = m_rp[i]; e < m_rp[i + 1]; e++) {
          const int d = std::abs(i - m_ci[e]);
          if (d >= lo && d < hi) bv[c[d]++] = m_val[e];
        }
    }
  };
  auto lower = [&](int g) {
    do g--; while (g > 0 && gstart[g] == gstart[g + 1]);
    return g;
  };
  // where the walk stops on the double sums
  int filled = nd;
  {
    double tot = 0.0;
    for (int d = 0; d < nd; d++) tot += gsq[d];
    const double keep_a = (1.0 - (double)frac) * tot;
    double kept_a = tot;
    int g = lower(nd);
    while (g > max_bw) {
      kept_a -= gsq[g];
      g = lower(g);
    }
    if (kept_a >= keep_a)
      while (g > 0 && kept_a - gsq[g] >= keep_a) {
        kept_a -= gsq[g];
        g = lower(g);
      }
    constexpr int kSlack = 8;  // groups placed below the predicted stop
    filled = std::max(0, g - kSlack);
    // SAPB_DROPOFF_PLACE=all places every group first, =none none (the
    // walk then places them when it reaches the first): both only for tests
    const char* env = std::getenv("SAPB_DROPOFF_PLACE");
    if (env && std::string(env) == "all") filled = 0;
    if (env && std::string(env) == "none") filled = nd;
    if (filled < nd) place(filled, nd);
  }
  auto need = [&](int g) {  // group g's values placed
    if (g < filled) {
      place(0, filled);
      filled = 0;
    }
  };
  squares.join();
  const T keep_min = (T(1) - frac) * total;
  T kept = total;
  // walk the groups from the longest distance down, summing squares from
  // the end of the list backwards (the reference's order)
  int g = lower(nd);  // the top non-empty group
  int kres = g;
  {
    T s = T(0);
    while (g > max_bw) {
      need(g);
      for (int p = gstart[g + 1] - 1; p >= gstart[g]; p--) s = s + bv[p] * bv[p];
      g = lower(g);
    }
    kept -= s;
    kres = g;
  }
  if (kept >= keep_min) {
    for (;;) {
      const int d = g;
      if (d == 0) { kres = 0; break; }
      need(g);
      T band = T(0);
      for (int p = gstart[g + 1] - 1; p >= gstart[g]; p--) band = band + bv[p] * bv[p];
      if (kept - band < keep_min) break;
      kept -= band;
      kres = d;
      g = lower(g);
    }
  }
  drop_actual = T(1) - kept / total;
  // kept: every entry within distance g, by row and, inside a row, by
  // decreasing column: the reference counting-sorts the kept list by column,
  // then places it by row in a forward pass that fills each row from its end
  // (graph.h:705-733)
  const int dkeep = g;
  tmp_rp.swap(m_rp);
  tmp_ci.swap(m_ci);
  tmp_val.swap(m_val);
  const std::vector<int>& rp0 = tmp_rp;
  const std::vector<int>& ci0 = tmp_ci;
  const std::vector<T>& v0 = tmp_val;
  m_rp.assign(n + 1, 0);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    int c = 0;
    for (int e = rp0[i]; e < rp0[i + 1]; e++) c += std::abs(i - ci0[e]) <= dkeep;
    m_rp[i + 1] = c;
  }
  prefix_sum(m_rp.data(), n);
  m_ci.resize(m_rp[n]);
  m_val.resize(m_rp[n]);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    const int a = m_rp[i];
    int w = a;
    bool ascending = true;
    for (int e = rp0[i]; e < rp0[i + 1]; e++) {
      if (std::abs(i - ci0[e]) > dkeep) continue;
      ascending = ascending && (w == a || m_ci[w - 1] < ci0[e]);
      m_ci[w] = ci0[e];
      m_val[w++] = v0[e];
    }
    // decreasing column order (the columns of a row are distinct, so the
    // order is unique): a row kept in increasing order is reversed, any
    // other sorted by insertion
    if (ascending) {
      std::reverse(m_ci.begin() + a, m_ci.begin() + w);
      std::reverse(m_val.begin() + a, m_val.begin() + w);
    } else {
      for (int q = a + 1; q < w; q++) {
        const int c = m_ci[q];
        const T x = m_val[q];
        int t = q;
        for (; t > a && m_ci[t - 1] < c; t--) {
          m_ci[t] = m_ci[t - 1];
          m_val[t] = m_val[t - 1];
        }
        m_ci[t] = c;
        m_val[t] = x;
      }
    }
  }
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
  couples_right.assign(n, 0);
  d_rp.assign(n + 1, 0);
  // per row: entries inside its partition (d_rp) and coupling entries
  // (ocnt), then row offsets, then the entries in row order
  std::vector<int>& ocnt = ws_i1;
  ocnt.assign(n + 1, 0);
  // partition p holds rows [first(p), first(p + 1)): an entry inside its
  // row's partition needs no division
  auto first = [&](int p) { return p * q + std::min(p, rem); };
#pragma omp parallel for schedule(static)
  for (int j = 0; j < n; j++) {
    const int pr = partition_of(j, q, rem), lo = first(pr), hi = first(pr + 1);
    int dc = 0, oc = 0;
    char right = 0;
    for (int e = m_rp[j]; e < m_rp[j + 1]; e++) {
      const int l = m_ci[e];
      if (l >= lo && l < hi) {
        dc++;
      } else {
        oc++;
        right |= (char)(l >= hi);
      }
    }
    d_rp[j + 1] = dc;
    ocnt[j + 1] = oc;
    couples_right[j] = right;
  }
  prefix_sum(d_rp.data(), n);
  prefix_sum(ocnt.data(), n);
  d_ci.resize(d_rp[n]);
  d_val.resize(d_rp[n]);
  offd_idx.resize(ocnt[n]);
  offd_val.resize(ocnt[n]);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < n; j++) {
    const int pr = partition_of(j, q, rem), lo = first(pr), hi = first(pr + 1);
    int dw = d_rp[j], ow = ocnt[j];
    for (int e = m_rp[j]; e < m_rp[j + 1]; e++) {
      const int l = m_ci[e];
      if (l >= lo && l < hi) {
        d_ci[dw] = l;
        d_val[dw++] = m_val[e];
        continue;
      }
      const int pc = partition_of(l, q, rem);
      if (pc > pr) {
        const int row_end = q * pr + (pr < rem ? pr + q + 1 : rem + q);
        const int col_start = q * pc + (pc < rem ? pc : rem);
        offd_idx[ow] = (long long)(pr * 2 * KK + (size_t)(j + K - row_end) * K + (l - col_start));
        offd_val[ow++] = m_val[e];
      } else {
        const int row_start = q * pr + (pr < rem ? pr : rem);
        const int col_end = q * pc + (pc < rem ? pc + q + 1 : rem + q);
        offd_idx[ow] = (long long)((pc * 2 + 1) * KK + (size_t)(j - row_start) * K + (l - col_end + K));
        offd_val[ow++] = m_val[e];
      }
    }
  }
}

// Second-level reordering (secondLevelReordering + partitionedRCM,
// graph.h:908-1008, 1593-1757): RCM inside every partition with the
// symmetrised-topology degree as BFS priority, up to 5 trials stopped by the
// level-growth rule or a bandwidth <= 128; then the diagonal matrix is
// permuted and first_rows computed.
template <typename T>
void Pipeline<T>::second_level(int K, int P) {
  const int q = n / P, rem = n % P;
  pfill(second_order, n, 0);
  pfill(second_pos, n, 0);
  std::vector<int>& order = pfill(bfs_order, n, 0);
  // the parallel pass keeps each partition's BFS state in the ranges of
  // shared arrays (its trials never leave its nodes); the serial replay
  // uses fresh whole-size arrays per partition
  std::vector<char>& tried_sh = pfill(bfs_tried, n, (char)0);
  std::vector<int>& pushed_sh = pfill(bfs_pushed, n, -1);
  std::vector<int>& level_sh = pfill(bfs_level, n, 0);
  std::vector<int> pnb(P + 1, 0);
  for (int p = 0; p < P; p++) pnb[p + 1] = pnb[p] + q + (p < rem ? 1 : 0);
  if ((int)part_scratch.size() < P) part_scratch.resize(P);
  // One partition.  Returns false, in the parallel pass, when a trial root
  // leaves the partition (the reference's root search walks on to the next
  // index): that trial's writes reach another partition, so every partition
  // is then redone serially in order, as the reference does.
  auto part = [&](int p, bool serial) -> bool {
    const int nb = pnb[p], ne = pnb[p + 1];
    for (int i = nb; i < ne; i++) second_order[i] = i;
    int best_bw = 0;
    for (int i = nb; i < ne; i++)
      for (int e = d_rp[i]; e < d_rp[i + 1]; e++) best_bw = std::max(best_bw, std::abs(i - d_ci[e]));
    PartScratch& sc = part_scratch[p];
    std::vector<int>& off = sc.off;
    std::vector<int>& adj = sc.adj;
    const int obase = serial ? 0 : nb;
    symmetric_adjacency(d_rp, d_ci, nb, ne, n, off, adj, obase, sc.pos);
    // row lengths of the partition's nodes as the reference computes them:
    // its transform covers row_offsets[nb+1 .. ne), one element short, so the
    // partition's last node keeps degree 0 (graph.h:1622-1625), which makes
    // it the first trial's root unless a node has no entries at all
    std::vector<int>& rowlen = sc.rowlen;
    rowlen.assign(ne - nb, 0);
    for (int i = nb; i < ne - 1; i++) rowlen[i - nb] = d_rp[i + 1] - d_rp[i];
    std::vector<char> tried_own;
    std::vector<int> pushed_own, level_own;
    if (serial) {
      tried_own.assign(n, 0);
      pushed_own.assign(n, -1);
      level_own.assign(n, 0);
    }
    std::vector<char>& tried = serial ? tried_own : tried_sh;
    std::vector<int>& pushed = serial ? pushed_own : pushed_sh;
    std::vector<int>& level = serial ? level_own : level_sh;
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
        if (serial) {
          while (tried[root]) root = (root + 1) % n;
        } else {  // the same walk, ending at the partition's end
          while (root < ne && tried[root]) root++;
        }
      }
      if (!serial && (root < nb || root >= ne)) return false;
      tried[root] = 1;
      // an order that cannot lower the bandwidth is given up early; the
      // trial still yields its levels for the stopping rule and next root
      bool gave_up = false;
      if (!cm_bfs(root, nb, ne, trial, off, adj, nullptr, pushed, level, order, last_level, obase, sc.fifo, best_bw,
                  &gave_up))
        break;
      if (!gave_up) {
        for (int k = nb; k < ne; k++) second_pos[order[k]] = k;
        int bw = 0;
        for (int i = nb; i < ne; i++) {
          const int pi = second_pos[i];
          for (int e = d_rp[i]; e < d_rp[i + 1]; e++) bw = std::max(bw, std::abs(pi - second_pos[d_ci[e]]));
        }
        if (best_bw > bw) {
          best_bw = bw;
          std::copy(order.begin() + nb, order.begin() + ne, second_order.begin() + nb);
        }
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
  tmp_rp.swap(d_rp);
  tmp_ci.swap(d_ci);
  tmp_val.swap(d_val);
  permute_rows(n, tmp_rp, tmp_ci, tmp_val, second_order, &second_pos, d_rp, d_ci, d_val);
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
#pragma omp parallel
  {
    std::vector<int> kp(P, 0);
    // the diagonal blocks' entries lie in their row's partition: one
    // division per row (the range test keeps any other entry exact)
    auto first = [&](int p) { return p * q + std::min(p, rem); };
#pragma omp for schedule(static) nowait
    for (int j = 0; j < n; j++) {
      const int pr = partition_of(j, q, rem), lo = first(pr), hi = first(pr + 1);
      for (int e = d_rp[j]; e < d_rp[j + 1]; e++) {
        const int l = d_ci[e];
        const int p = (l >= lo && l < hi) ? pr : partition_of(l, q, rem);
        kp[p] = std::max(kp[p], std::abs(l - j));
      }
    }
#pragma omp critical
    for (int p = 0; p < P; p++) part_k[p] = std::max(part_k[p], kp[p]);
  }
}

// The whole sparse setup of transformToBandedMatrix (precond.h:1656-2101)
// up to the band layout.
template <typename T>
void Pipeline<T>::run(const double* weight, const double* rowmax) {
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
  int kdb = 0;
#pragma omp parallel for schedule(static) reduction(max : kdb)
  for (int i = 0; i < n; i++)
    for (int e = m_rp[i]; e < m_rp[i + 1]; e++) kdb = std::max(kdb, std::abs(i - m_ci[e]));
  k_db = kdb;
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
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; k++) {
    final_order[k] = rcm_order[second_order[k]];
    final_pos[k] = second_pos[rcm_pos[db_row_perm[k]]];
  }
  lap("compose");
}

template class Pipeline<float>;
template class Pipeline<double>;

}  // namespace rp

void set_last_error(const std::string& msg);

namespace {

// stage times of the calling thread's last sap_reorder_host
thread_local std::vector<std::pair<const char*, double>> g_last_stages;

// The host part of a CSR setup on its own: explicit zeros removed in T,
// DB weights log(rowmax / |a|) computed on the host (std::log), the
// pipeline, and its outputs copied out.
template <typename T>
int reorder_host(int n, int nnz, const int* rp, const int* ci, const double* v, int P, const sap_options& o,
                 sap_reorder_info* info, int* db_row_perm, int* final_pos, int* final_order, int* first_rows,
                 int* part_k) {
  rp::Pipeline<T> pl;
  pl.n = n;
  pl.P_req = P;
  pl.do_db = o.performDB != 0;
  pl.scale = o.applyScaling != 0;
  pl.drop_frac = o.dropOffFraction;
  pl.max_bandwidth = o.maxBandwidth;
  pl.var_band = o.variableBandwidth != 0;
  // (row-parallel: count, prefix, fill; then the weights per row)
  pl.in_rp.assign(n + 1, 0);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    int c = 0;
    for (int e = rp[i]; e < rp[i + 1]; e++) c += (T)v[e] != T(0);
    pl.in_rp[i + 1] = c;
  }
  rp::prefix_sum(pl.in_rp.data(), n);
  pl.in_ci.resize(pl.in_rp[n]);
  pl.in_val.resize(pl.in_rp[n]);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; i++) {
    int d = pl.in_rp[i];
    for (int e = rp[i]; e < rp[i + 1]; e++)
      if ((T)v[e] != T(0)) {
        pl.in_ci[d] = ci[e];
        pl.in_val[d++] = (T)v[e];
      }
  }
  pl.nnz = (int)pl.in_ci.size();
  std::vector<double> w, rmax;
  if (pl.do_db) {
    w.resize(pl.nnz);
    rmax.resize(n);
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; i++) {
      double m = 0.0;
      for (int e = pl.in_rp[i]; e < pl.in_rp[i + 1]; e++) m = std::max(m, std::fabs((double)pl.in_val[e]));
      rmax[i] = m;
      for (int e = pl.in_rp[i]; e < pl.in_rp[i + 1]; e++) w[e] = std::log(m / std::fabs((double)pl.in_val[e]));
    }
  }
  pl.run(w.data(), rmax.data());
  g_last_stages = pl.stage_ms;
  info->K = pl.K;
  info->P = pl.P;
  info->k_db = pl.k_db;
  info->k_reorder = pl.k_reorder;
  info->var_band = pl.var_band ? 1 : 0;
  info->drop_actual = (double)pl.drop_actual;
  if (db_row_perm) std::copy(pl.db_row_perm.begin(), pl.db_row_perm.end(), db_row_perm);
  if (final_pos) std::copy(pl.final_pos.begin(), pl.final_pos.end(), final_pos);
  if (final_order) std::copy(pl.final_order.begin(), pl.final_order.end(), final_order);
  if (first_rows) std::copy(pl.first_rows.begin(), pl.first_rows.end(), first_rows);
  if (part_k) {  // a constant band has K in every partition
    if (pl.var_band) std::copy(pl.part_k.begin(), pl.part_k.end(), part_k);
    else std::fill(part_k, part_k + pl.P, pl.K);
  }
  return SAP_OK;
}

}  // namespace
}  // namespace sapb

extern "C" int sap_reorder_host(int n, int nnz, const int* rp, const int* ci, const double* v, int num_partitions,
                                const sap_options* opts, int prec_dtype, int threads, sap_reorder_info* info,
                                int* db_row_perm, int* final_pos, int* final_order, int* first_rows, int* part_k) {
  using namespace sapb;
  if (n <= 0 || nnz < 0 || !rp || !ci || !v || !opts || !info || num_partitions < 1 ||
      (prec_dtype != SAP_PREC_FLOAT && prec_dtype != SAP_PREC_DOUBLE)) {
    set_last_error("invalid arguments to sap_reorder_host");
    return SAP_ERR_INVALID_ARGUMENT;
  }
  if (rp[0] != 0 || rp[n] != nnz) {
    set_last_error("row offsets inconsistent with nnz");
    return SAP_ERR_INVALID_ARGUMENT;
  }
  int bad_rp = 0, bad_ci = 0;
#pragma omp parallel for schedule(static) reduction(| : bad_rp)
  for (int i = 0; i < n; i++) bad_rp |= rp[i] > rp[i + 1];
  if (bad_rp) {
    set_last_error("row offsets not monotone");
    return SAP_ERR_INVALID_ARGUMENT;
  }
#pragma omp parallel for schedule(static) reduction(| : bad_ci)
  for (int e = 0; e < nnz; e++) bad_ci |= ci[e] < 0 || ci[e] >= n;
  if (bad_ci) {
    set_last_error("column index out of range");
    return SAP_ERR_INVALID_ARGUMENT;
  }
  const int saved = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  int rc = SAP_OK;
  try {
    rc = prec_dtype == SAP_PREC_DOUBLE
             ? reorder_host<double>(n, nnz, rp, ci, v, num_partitions, *opts, info, db_row_perm, final_pos,
                                    final_order, first_rows, part_k)
             : reorder_host<float>(n, nnz, rp, ci, v, num_partitions, *opts, info, db_row_perm, final_pos,
                                   final_order, first_rows, part_k);
  } catch (const Error& e) {
    set_last_error(e.what());
    rc = e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    rc = SAP_ERR_INVALID_ARGUMENT;
  }
  if (threads > 0) omp_set_num_threads(saved);
  return rc;
}

extern "C" int sap_reorder_host_stages(int cap, const char** names, double* ms, int* count) {
  using namespace sapb;
  if (!count || cap < 0) {
    set_last_error("invalid arguments to sap_reorder_host_stages");
    return SAP_ERR_INVALID_ARGUMENT;
  }
  *count = (int)g_last_stages.size();
  for (int i = 0; i < cap && i < *count; i++) {
    if (names) names[i] = g_last_stages[i].first;
    if (ms) ms[i] = g_last_stages[i].second;
  }
  return SAP_OK;
}
