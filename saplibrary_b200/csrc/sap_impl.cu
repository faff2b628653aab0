// Host orchestration of the B200 SPIKE solver and its C ABI (include/sap_b200.h).
//
// One solver = one CUDA stream.  Setup builds the partitioned band on the
// device, factors it, computes the spike tips, the reduced system and the
// chunk transfer matrices of the parallel sweeps; solve runs the
// reference's BiCGStab(L) (sap/bicgstab2.h:32-360) with its monitor
// (sap/monitor.h:154-339) over FP64 device vectors.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "krylov_kernels.cuh"
#include "precond_kernels.cuh"
#include "reorder.h"
#include "reorder_pipeline.h"
#include "wide_host.cuh"

namespace sapb {

std::atomic<int64_t> g_launches{0};
std::atomic<int64_t> g_lib_calls{0};
static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

// --- live kernel profiling -----------------------------------------------------
struct ProfState {
  std::mutex mu;
  std::string name;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pairs;
};
static ProfState g_prof;

ProfScope::ProfScope(const char* name, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(g_prof.mu);
  if (g_prof.name.empty() || g_prof.name != name) return;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return;
  on = true;
  s = st;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s);
}
ProfScope::~ProfScope() {
  if (!on) return;
  cudaEventRecord(b, s);
  std::lock_guard<std::mutex> lk(g_prof.mu);
  g_prof.pairs.emplace_back(a, b);
}

static int grid_for(long long n, int threads, int cap = 148 * 16) {
  long long g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

using Clock = std::chrono::steady_clock;
static double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// ---------------------------------------------------------------------------
struct Banded {
  int n = 0, K = 0;
  DBuf<double> A;  // row-major band on the device
};

struct Csr {
  int n = 0, nnz = 0;
  // host copies (reordering runs on the host), page-locked blocks from a
  // pool: the uploads run at full speed and repeated copies reuse warm
  // pages.  Declared before the device buffers, so that they go back to the
  // pool only after those are freed (cudaFree waits for copies in flight).
  PinnedHostVec<int> rp_h, ci_h;
  PinnedHostVec<double> v_h;
  DBuf<int> rp, ci;
  DBuf<double> v;
  DBuf<int> blk;  // row blocks of k_spmv_csr_blocks
  int nblk = 0;
};

struct Spmv {
  int kind = 0;  // 0 banded, 1 csr, 2 callback
  const Banded* band = nullptr;
  const Csr* csr = nullptr;
  sap_spmv_fn fn = nullptr;
  void* ctx = nullptr;
  int n = 0;
  void apply(const double* x, double* y, cudaStream_t s) const {
    if (kind == 0) {
      SAPB_PROF("spmv_banded", s);
      k_spmv_banded<<<grid_for((long long)band->n * 32, 256, 148 * 32), 256, 0, s>>>(band->A.get(), x, y, band->n, band->K);
      SAPB_LAUNCHED();
    } else if (kind == 1) {
      SAPB_PROF("spmv_csr", s);
      k_spmv_csr_blocks<<<csr->nblk, kSpmvRows, 0, s>>>(csr->blk.get(), csr->rp.get(), csr->ci.get(), csr->v.get(),
                                                         x, y);
      SAPB_LAUNCHED();
    } else {
      fn(ctx, x, y, (void*)s);
    }
  }
};

// ---------------------------------------------------------------------------
// Preconditioner (sap::Precond, sap/precond.h).  PrecBase holds what does not
// depend on the value type; PrecondT<T> is the Precond<PrecVector> of a
// float or double PrecValueType (sap/solver.h:153).
class PrecBase {
 public:
  sap_options o{};
  int P_req = 1;
  cudaStream_t st = nullptr;

  int n = 0, K = 0, P = 1;
  bool spike = false, lu_ul = false;
  bool tf32 = false;  // wide-band block products in TF32 (FP32 storage)
  bool h16 = false;   // wide-band block sweeps over FP16 block-scaled copies
  int ptype = SAP_PRECOND_SPIKE;
  std::vector<PartDev> parts_h;
  DBuf<PartDev> parts_d;

  // reordering (sparse path): permutations, interface map, statistics
  bool reordered = false;
  bool var_band = false;
  DBuf<int> gin_d, sout_d, iface_d, partcol_d;
  std::vector<int> final_pos_h, final_order_h, db_row_perm_h, first_rows_h, part_k_h;

  // statistics
  double t_toBanded = 0, t_offDiags = 0, t_bandLU = 0, t_assembly = 0, t_fullLU = 0, t_transfer = 0;
  double t_reorder = 0, t_dropOff = 0, t_cpu_assemble = 0, t_DB = 0;
  double t_pipeline = 0;  // the whole host pipeline
  int k_reorder = 0, k_db = 0;
  double drop_actual = 0;

  virtual ~PrecBase() {}
  // Band setups: the row-major FP64 band of a BandedMatrix, or a CSR matrix
  // used without reordering.
  virtual void setup_rowmajor(const double* A_dev, int n_, int K_) = 0;
  virtual void setup_csr_direct(const Csr& A, int K_) = 0;
  virtual void setup_sparse(const Csr& A) = 0;
  virtual void apply_band(const double* v, double* z) = 0;
  virtual void block_layout(int& bs, int& nb) const = 0;
  // raise the errors device waits recorded (call after a stream synchronisation)
  virtual void check_device() = 0;
  virtual void update_values(const double* entries, long long nnz, bool device) = 0;
  void apply(const double* v, double* z) { apply_band(v, z); }

  void clamp_partitions_banded() {
    // convertToBandedMatrix (sap/precond.h:2116-2117, 2258-2259)
    int maxP = std::max(1, n / std::max(K + 1, 2 * K));
    P = std::min(P_req, maxP);
  }
  void init_parts_const() {
    parts_h.resize(P);
    int q = n / P, r = n % P;
    for (int p = 0; p < P; p++) {
      PartDev d{};
      d.start = p * q + std::min(p, r);
      d.size = q + (p < r ? 1 : 0);
      d.K = K;
      d.ul = (lu_ul && p == P - 1) ? 1 : 0;
      d.boff = (long long)d.start * (2 * K + 1);
      parts_h[p] = d;
    }
    parts_d.upload(parts_h, st);
  }
  int parts_maxK() const {
    int m = 0;
    for (auto& p : parts_h) m = std::max(m, p.K);
    return m;
  }
};

template <typename T>
class PrecondT : public PrecBase {
 public:
  DBuf<T> B, B2, offd, V, W, S, scratch;
  // chunked sweeps
  std::vector<ChunkDev> chunks_h;
  DBuf<ChunkDev> chunks_d;
  DBuf<long long> koff_d, toff_d;
  DBuf<int> first1_d, first2_d, pchunk0_d, pnchunk_d;
  DBuf<T> T1, T2, tails1, tails2, carry1, carry2;
  DBuf<T> F, Gv, Y;
  DBuf<T> sin_d, cout_d;  // DB row / column scales in band order (reordered path)
  // TF32 forms without reordering: power-of-two diagonal scales (band order),
  // the factors being those of S A S; the apply scales its input and output by S
  DBuf<T> dscale;
  bool dscaled = false;
  const T* in_scale() const { return reordered ? sin_d.get() : (dscaled ? dscale.get() : nullptr); }
  const T* out_scale() const { return reordered ? cout_d.get() : (dscaled ? dscale.get() : nullptr); }
  DBuf<int> flag;
  int maxChunk = 0, sweepThreads = 32, scanG = 1;
  // Numeric inputs of a CSR setup, on the device: the entries of the
  // partitions' diagonal blocks (band rows / columns, values; for a constant
  // band, all entries) and the coupling entries (index into the dense
  // coupling blocks, values).  update() rewrites the values and reruns the
  // numeric phase from them.
  DBuf<int> co_row, co_col;
  DBuf<T> co_val;
  DBuf<long long> cp_idx;
  DBuf<T> cp_val;
  size_t cp_size = 0;
  std::vector<int> iface_h;
  // update() maps (trackReordering): the input entry of every diagonal-block
  // and coupling entry and its DB scale factor (graph.h:1292-1330 scaleMap,
  // bandedMatMap / offDiagMap of graph.h:795-886, 1031-1062, 1140-1184)
  DBuf<int> co_src, cp_src;
  DBuf<T> co_scale, cp_scale;
  int numeric_kind = 0;  // 0: no CSR numeric phase, 1: variable band, 2: constant band

  std::unique_ptr<WideBand<T>> wide;  // block (GEMM) path of wide bands (buffers kept across setups)
  bool wide_active = false;           // the last setup used the block path
  void block_layout(int& bs, int& nb) const override {
    bs = wide_active ? wide->bs : 0;
    nb = wide_active ? wide->nb : 0;
  }

  // Partitions are factored and applied as block tridiagonal (wide_host.cuh)
  // when the narrow factor's window (K+1+8 band columns of 2K+1 values) does
  // not fit in 200 KB of shared memory, where the narrow kernels fall back to
  // a global-memory window and the block path is faster (FP64 from K ~ 108,
  // FP32 from K ~ 155 on B200), and always above K = 1024.  The environment
  // variable SAPB_WIDE_MIN_K sets an explicit threshold instead.
  static bool use_wide(int kmax) {
    if (kmax > 1024) return true;
    const char* e = std::getenv("SAPB_WIDE_MIN_K");
    const int v = e ? std::atoi(e) : 0;
    if (v > 0) return kmax >= v;
    constexpr int D = 8;
    const size_t smem = ((size_t)(kmax + 1 + D) * (2 * kmax + 1) + (kmax + 1 + D)) * sizeof(T);
    return smem > 200 * 1024;
  }

  // Boosting of the band factorization (partBandedLU and its variants,
  // sap/precond.h:3882-3983): the variable-band kernels always boost; the
  // constant-band kernels boost for K >= 70 (with more than one partition
  // when decoupled) or when safeFactorization is set.
  bool factor_boost() const {
    if (var_band) return true;
    if (!spike) return o.safeFactorization || (P > 1 && K >= 70);
    return o.safeFactorization || K >= 70;
  }

  void wide_check_memory(int kmax) {
    size_t fr = 0, tot = 0;
    SAPB_CUDA(cudaMemGetInfo(&fr, &tot));
    if (wide) fr += wide->bytes_held();  // reused (or released) by the new setup
    const double need = WideBand<T>::factor_bytes(n, P, kmax, h16 && sizeof(T) == 4,
                                                  tf32 && sizeof(T) == 4 && WideBand<T>::tc_gemm_enabled());
    if (need > 0.92 * (double)fr)
      throw Error(SAP_ERR_OUT_OF_MEMORY, "wide-band factors need " + std::to_string(need / 1e9) + " GB, " +
                                             std::to_string((double)fr / 1e9) + " GB free");
  }

  // Interface unknowns of the variable band: the last K first-level rows of
  // partition i and the first K of partition i+1, in band (second-level) order.
  std::vector<int> var_iface(const rp::Pipeline<T>& pl) const {
    std::vector<int> iface((size_t)(P - 1) * 2 * K);
    for (int i = 0; i < P - 1; i++) {
      const int e_i = parts_h[i].start + parts_h[i].size, s1 = parts_h[i + 1].start;
      for (int k = 0; k < K; k++) {
        iface[(size_t)i * 2 * K + k] = pl.second_pos[e_i - K + k];
        iface[(size_t)i * 2 * K + K + k] = pl.second_pos[s1 + k];
      }
    }
    return iface;
  }

  void wide_init(int kmax) {
    wide_check_memory(kmax);
    std::vector<int> ps(P), pz(P);
    for (int p = 0; p < P; p++) {
      ps[p] = parts_h[p].start;
      pz[p] = parts_h[p].size;
    }
    if (!wide) wide = std::make_unique<WideBand<T>>();
    wide->init(st, n, WideBand<T>::block_size(kmax, tf32 && sizeof(T) == 4 && WideBand<T>::tc_gemm_enabled()), ps, pz,
               tf32, h16);
    wide_active = true;
  }

  // spikes and reduced system of the block path (offd: the row-major
  // coupling blocks on the device, kept for the next setup of the same
  // layout: at the 1M-row workload it is 1.2 GB, whose allocation and
  // release every setup cost a device synchronisation each)
  void wide_couple(const std::vector<int>& iface) {
    auto t0 = Clock::now();
    wide->spikes(offd.get(), iface, K);
    t_assembly = ms_since(t0);
    t0 = Clock::now();
    wide->reduced(offd.get(), iface, o.safeFactorization != 0);
    t_fullLU = ms_since(t0);
  }

  void setup_rowmajor(const double* A_dev, int n_, int K_) override {
    numeric_kind = 0;
    n = n_;
    K = K_;
    clamp_partitions_banded();
    B.alloc((size_t)(2 * K + 1) * n);
    auto t1 = Clock::now();
    k_band_from_rowmajor<T><<<grid_for((long long)(2 * K + 1) * n, 256, 148 * 32), 256, 0, st>>>(A_dev, B.get(), n, K);
    SAPB_LAUNCHED();
    SAPB_CUDA(cudaStreamSynchronize(st));
    t_toBanded = ms_since(t1);
    setup_from_band();
  }

  void setup_csr_direct(const Csr& A, int K_) override {
    n = A.n;
    K = K_;
    numeric_kind = 0;
    clamp_partitions_banded();
    B.alloc((size_t)(2 * K + 1) * n);
    B.zero(st);
    auto t1 = Clock::now();
    k_band_from_csr<T><<<grid_for(n, 256), 256, 0, st>>>(A.rp.get(), A.ci.get(), A.v.get(), B.get(), n, K);
    SAPB_LAUNCHED();
    SAPB_CUDA(cudaStreamSynchronize(st));
    t_toBanded = ms_since(t1);
    if (o.trackReordering) {
      // band position (i, j) of every entry, scale 1 (convertToBandedMatrix
      // of a CSR matrix, precond.h:2240-2368)
      std::vector<int> rows(A.nnz), src(A.nnz);
      for (int i = 0; i < n; i++)
        for (int e = A.rp_h[i]; e < A.rp_h[i + 1]; e++) rows[e] = i;
      for (int e = 0; e < A.nnz; e++) src[e] = e;
      co_row.upload(rows, st);
      co_col.upload(A.ci_h.data(), A.ci_h.size(), st);
      co_src.upload(src, st);
      co_scale.upload(std::vector<T>(A.nnz, T(1)), st);
      co_val.alloc(A.nnz);
      cp_idx.release();
      cp_val.release();
      cp_src.release();
      cp_scale.release();
      cp_size = 0;
      numeric_kind = 2;
    }
    setup_from_band();
  }

  // Band from the diagonal-block entries, then the constant-band setup.
  void numeric_const() {
    B.alloc((size_t)(2 * K + 1) * n);
    B.zero(st);
    const long long m = (long long)co_row.size();
    if (m) {
      k_band_from_coo_const<T><<<grid1d(m), 256, 0, st>>>(co_row.get(), co_col.get(), co_val.get(), m, B.get(), K);
      SAPB_LAUNCHED();
    }
    SAPB_CUDA(cudaStreamSynchronize(st));
    setup_from_band();
  }

  // Dense coupling blocks from the coupling entries.
  void coupling_dense() {
    offd.alloc(cp_size);
    offd.zero(st);
    const long long m = (long long)cp_idx.size();
    if (m) {
      k_scatter_idx<T><<<grid1d(m), 256, 0, st>>>(cp_idx.get(), cp_val.get(), m, offd.get());
      SAPB_LAUNCHED();
    }
    SAPB_CUDA(cudaStreamSynchronize(st));
  }

  // Precond::update (sap/precond.h:751-900): values = entries x scaleMap,
  // scattered through the maps of the setup, then the numeric phase again.
  void update_values(const double* entries, long long nnz_in, bool device) override {
    if (numeric_kind == 0 || co_src.size() != co_row.size())
      throw Error(SAP_ERR_UNSUPPORTED, "update() needs a CSR setup with trackReordering");
    DBuf<double> ev;
    const double* e = entries;
    if (!device) {
      ev.upload(entries, (size_t)nnz_in, st);
      e = ev.get();
    }
    const long long m1 = (long long)co_src.size(), m2 = (long long)cp_src.size();
    if (m1) {
      k_gather_scale<T><<<grid1d(m1), 256, 0, st>>>(e, co_src.get(), co_scale.get(), m1, co_val.get());
      SAPB_LAUNCHED();
    }
    if (m2) {
      k_gather_scale<T><<<grid1d(m2), 256, 0, st>>>(e, cp_src.get(), cp_scale.get(), m2, cp_val.get());
      SAPB_LAUNCHED();
    }
    SAPB_CUDA(cudaStreamSynchronize(st));
    t_reorder = t_DB = t_dropOff = t_transfer = 0;
    if (numeric_kind == 1) numeric_var();
    else numeric_const();
  }

  // transformToBandedMatrix (sap/precond.h:1656-2101) and the rest of the
  // setup for a CSR matrix with reordering: DB weights on the device, the
  // graph pipeline on the host, then the band, factors, spikes and sweeps on
  // the device.
  void setup_sparse(const Csr& A) override {
    if (o.dbFirstStageOnly) throw Error(SAP_ERR_UNSUPPORTED, "dbFirstStageOnly is not supported");
    if (o.ilu_level >= 0) throw Error(SAP_ERR_UNSUPPORTED, "ILU preconditioning is out of scope");
    wide_active = false;
    auto t0 = Clock::now();
    n = A.n;
    if (!pipe) pipe = std::make_unique<rp::Pipeline<T>>();
    rp::Pipeline<T>& pl = *pipe;
    pl.n = n;
    pl.P_req = P_req;
    pl.do_db = o.performDB != 0;
    pl.scale = o.applyScaling != 0;
    pl.drop_frac = o.dropOffFraction;
    pl.max_bandwidth = o.maxBandwidth;
    pl.var_band = o.variableBandwidth != 0;
    // the matrix in the preconditioner's value type, explicit zeros removed
    // (row-parallel: count, prefix, fill)
    pl.in_rp.assign(n + 1, 0);
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; i++) {
      int c = 0;
      for (int e = A.rp_h[i]; e < A.rp_h[i + 1]; e++) c += (T)A.v_h[e] != T(0);
      pl.in_rp[i + 1] = c;
    }
    rp::prefix_sum(pl.in_rp.data(), n);
    pl.in_ci.resize(pl.in_rp[n]);
    pl.in_val.resize(pl.in_rp[n]);
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; i++) {
      int d = pl.in_rp[i];
      for (int e = A.rp_h[i]; e < A.rp_h[i + 1]; e++) {
        const T a = (T)A.v_h[e];
        if (a != T(0)) {
          pl.in_ci[d] = A.ci_h[e];
          pl.in_val[d++] = a;
        }
      }
    }
    pl.nnz = (int)pl.in_ci.size();
    const double* w = nullptr;
    const double* rmax = nullptr;
    if (pl.do_db) {
      // weights from the matrix's device copy when no explicit zero was
      // removed (same entries in the same order), else from an upload of the
      // filtered host matrix; read back into page-locked buffers
      const bool same = pl.nnz == A.nnz;
      DBuf<int> drp;
      DBuf<double> da;
      const int* rpd = A.rp.get();
      const double* ad = A.v.get();
      if (!same) {
        std::vector<double>& av = db_av;
        av.resize(pl.in_val.size());
#pragma omp parallel for schedule(static, 65536)
        for (long long e = 0; e < (long long)av.size(); e++) av[e] = (double)pl.in_val[e];
        drp.upload(pl.in_rp, st);
        da.upload(av, st);
        rpd = drp.get();
        ad = da.get();
      }
      db_wd.alloc(pl.in_val.size());
      db_md.alloc(n);
      k_db_weights<<<grid_for((long long)n * 32, 256, 148 * 32), 256, 0, st>>>(
          rpd, ad, db_wd.get(), db_md.get(), n, (same && sizeof(T) == 4) ? 1 : 0);
      SAPB_LAUNCHED();
      double* wh = db_wh.reserve(pl.in_val.size());
      double* mh = db_mh.reserve(n);
      SAPB_CUDA(cudaMemcpyAsync(wh, db_wd.get(), pl.in_val.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      SAPB_CUDA(cudaMemcpyAsync(mh, db_md.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
      SAPB_CUDA(cudaStreamSynchronize(st));
      w = wh;
      rmax = mh;
    }
    t_transfer = ms_since(t0);
    auto t1 = Clock::now();
    pl.run(w, rmax);
    t_pipeline = ms_since(t1);
    // stage times as the reference's timers split them: DB, reordering
    // (RCM and the second level), drop-off; the rest is assembly
    t_DB = pl.stage("db");
    t_reorder = pl.stage("rcm") + pl.stage("second_level");
    t_dropOff = pl.stage("drop_off");
    k_db = pl.k_db;
    k_reorder = pl.k_reorder;
    drop_actual = (double)pl.drop_actual;
    K = pl.K;
    P = pl.P;
    var_band = pl.var_band;
    // the permutations kept for sap_solver_get_reorder (copied in parallel)
    auto keep = [](std::vector<int>& dst, const std::vector<int>& src) {
      dst.resize(src.size());
      const long long m = (long long)src.size();
#pragma omp parallel for schedule(static)
      for (int c = 0; c < 16; c++) std::copy(src.begin() + m * c / 16, src.begin() + m * (c + 1) / 16, dst.begin() + m * c / 16);
    };
    keep(final_pos_h, pl.final_pos);
    keep(final_order_h, pl.final_order);
    keep(db_row_perm_h, pl.db_row_perm);
    first_rows_h = pl.first_rows;
    part_k_h = pl.part_k;
    // leftTrans / rightTrans as gathers and scatters in band order, built in
    // a page-locked buffer kept across setups and uploaded asynchronously
    // (later synchronisations on the stream precede the buffer's reuse)
    {
      const size_t tw = ((size_t)n * sizeof(T) + sizeof(int) - 1) / sizeof(int);
      SAPB_CUDA(cudaStreamSynchronize(st));  // the previous setup's uploads from the buffer are done
      int* pin = gather_pin.reserve(2 * (size_t)n + 2 * tw);
      int* gin = pin;
      int* sout = pin + n;
      T* sn = reinterpret_cast<T*>(pin + 2 * (size_t)n);
      T* cn = reinterpret_cast<T*>(pin + 2 * (size_t)n + tw);
#pragma omp parallel for schedule(static, 4096)
      for (int q = 0; q < n; q++) {
        gin[pl.final_pos[q]] = q;
        sn[pl.final_pos[q]] = pl.scale ? (T)pl.row_scale[q] : T(1);
        sout[q] = pl.final_order[q];
        cn[q] = pl.scale ? (T)pl.col_scale[pl.final_order[q]] : T(1);
      }
      gin_d.upload(gin, n, st);
      sout_d.upload(sout, n, st);
      sin_d.upload(sn, n, st);
      cout_d.upload(cn, n, st);
    }
    reordered = true;
    if (!var_band) {
      // constant band over the whole reordered matrix (assembleBandedMatrix, graph.h:1019-1091)
      upload_coo(pl.m_rp, pl.m_ci, pl.m_val);
      cp_idx.release();
      cp_val.release();
      cp_size = 0;
      numeric_kind = 2;
      if (o.trackReordering) build_update_maps(A, pl);
      t_cpu_assemble = ms_since(t0) - t_transfer - t_DB - t_reorder - t_dropOff;
      numeric_const();
      return;
    }
    // variable band: partitions with their own K_p (>= 1 for storage)
    ptype = o.precondType;
    spike = (ptype == SAP_PRECOND_SPIKE && P > 1);
    lu_ul = false;  // a variable band forces LU_only (driver_test.cu:832-833)
    if (ptype == SAP_PRECOND_NONE) return;
    parts_h.resize(P);
    const int q = n / P, r = n % P;
    long long off = 0;
    for (int p = 0; p < P; p++) {
      PartDev d{};
      d.start = p * q + std::min(p, r);
      d.size = q + (p < r ? 1 : 0);
      d.K = std::max(1, pl.part_k[p]);
      d.ul = 0;
      d.boff = off;
      off += (long long)d.size * (2 * d.K + 1);
      parts_h[p] = d;
    }
    partcol_h.resize(n);
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < P; p++)
      std::fill(partcol_h.begin() + parts_h[p].start, partcol_h.begin() + parts_h[p].start + parts_h[p].size, p);
    parts_d.upload(parts_h, st);
    partcol_d.upload(partcol_h, st);
    boff_total = off;
    upload_coo(pl.d_rp, pl.d_ci, pl.d_val);
    cp_idx.upload(pl.offd_idx, st);
    cp_val.upload(pl.offd_val, st);
    cp_size = pl.offd_size;
    iface_h = spike ? var_iface(pl) : std::vector<int>();
    numeric_kind = 1;
    if (o.trackReordering) build_update_maps(A, pl);
    t_cpu_assemble = ms_since(t0) - t_transfer - t_DB - t_reorder - t_dropOff;
    numeric_var();
  }

  long long boff_total = 0;
  // host state kept across setups (its memory is reused, not re-faulted)
  std::unique_ptr<rp::Pipeline<T>> pipe;
  std::vector<double> db_av;
  DBuf<double> db_wd, db_md;          // DB weights and row maxima on the device
  PinnedBuf<double> db_wh, db_mh;     // and their page-locked host copies
  PinnedBuf<int> coo_pin;  // staging of the COO uploads
  PinnedBuf<int> gather_pin;  // staging of the band-order gathers and scales
  std::vector<int> partcol_h;  // partition of every band row (kept across setups)

  // device COO (band rows, columns, values) of a CSR in band order
  // (through a page-locked staging buffer: rows, columns and values are
  // packed into it in parallel, then copied in one transfer each)
  void upload_coo(const std::vector<int>& rp_, const std::vector<int>& ci_, const std::vector<T>& v_) {
    const size_t m = ci_.size();
    const size_t words = 2 * m + (m * sizeof(T) + sizeof(int) - 1) / sizeof(int);
    int* pin = coo_pin.reserve(words);
    int* prow = pin;
    int* pcol = pin + m;
    T* pval = reinterpret_cast<T*>(pin + 2 * m);
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; i++)
      for (int e = rp_[i]; e < rp_[i + 1]; e++) {
        prow[e] = i;
        pcol[e] = ci_[e];
        pval[e] = v_[e];
      }
    co_row.alloc(m);
    co_col.alloc(m);
    co_val.alloc(m);
    if (m) {
      SAPB_CUDA(cudaMemcpyAsync(co_row.get(), prow, m * sizeof(int), cudaMemcpyHostToDevice, st));
      SAPB_CUDA(cudaMemcpyAsync(co_col.get(), pcol, m * sizeof(int), cudaMemcpyHostToDevice, st));
      SAPB_CUDA(cudaMemcpyAsync(co_val.get(), pval, m * sizeof(T), cudaMemcpyHostToDevice, st));
    }
    // the staging buffer is reused by the next upload: finish these first
    SAPB_CUDA(cudaStreamSynchronize(st));
  }

  // update() maps: every input entry located in the setup's numeric inputs
  // (its position after DB, RCM, drop-off, the partition split and the
  // second-level reordering); dropped entries and explicit zeros have none.
  void build_update_maps(const Csr& A, const rp::Pipeline<T>& pl) {
    const int q = n / P, rem = n % P;
    auto part_of = [&](int x) { return x < rem * (q + 1) ? x / (q + 1) : rem + (x - rem * (q + 1)) / q; };
    const std::vector<int>& rp_ = var_band ? pl.d_rp : pl.m_rp;
    const std::vector<int>& ci_ = var_band ? pl.d_ci : pl.m_ci;
    std::vector<int> csrc(ci_.size(), -1), psrc(pl.offd_idx.size(), -1);
    std::vector<T> cscale(ci_.size(), T(1)), pscale(pl.offd_idx.size(), T(1));
    std::vector<std::pair<long long, int>> cpl(pl.offd_idx.size());
    for (size_t k = 0; k < cpl.size(); k++) cpl[k] = {pl.offd_idx[k], (int)k};
    std::sort(cpl.begin(), cpl.end());
    const long long KK = (long long)K * K;
    for (int i = 0; i < n; i++)
      for (int e = A.rp_h[i]; e < A.rp_h[i + 1]; e++) {
        if ((T)A.v_h[e] == T(0)) continue;  // removed before reordering (precond.h:1690-1713)
        const int j = A.ci_h[e];
        const T sc = pl.scale ? (T)(pl.row_scale[i] * pl.col_scale[j]) : T(1);
        const int i1 = pl.rcm_pos[pl.db_row_perm[i]], j1 = pl.rcm_pos[j];
        const int pr = part_of(i1), pc = part_of(j1);
        if (!var_band || pr == pc) {
          const int r2 = var_band ? pl.second_pos[i1] : i1, c2 = var_band ? pl.second_pos[j1] : j1;
          for (int t = rp_[r2]; t < rp_[r2 + 1]; t++)
            if (ci_[t] == c2) {
              csrc[t] = e;
              cscale[t] = sc;
              break;
            }
          continue;
        }
        long long idx = -1;
        if (pc == pr + 1) {
          const int row_end = q * pr + (pr < rem ? pr + q + 1 : rem + q);
          const int col_start = q * pc + (pc < rem ? pc : rem);
          const int a = i1 + K - row_end, c = j1 - col_start;
          if (a >= 0 && a < K && c >= 0 && c < K) idx = pr * 2 * KK + (long long)a * K + c;
        } else if (pr == pc + 1) {
          const int row_start = q * pr + (pr < rem ? pr : rem);
          const int col_end = q * pc + (pc < rem ? pc + q + 1 : rem + q);
          const int a = i1 - row_start, c = j1 - col_end + K;
          if (a >= 0 && a < K && c >= 0 && c < K) idx = (pc * 2 + 1) * KK + (long long)a * K + c;
        }
        if (idx < 0) continue;
        auto it = std::lower_bound(cpl.begin(), cpl.end(), std::make_pair(idx, -1));
        if (it != cpl.end() && it->first == idx) {
          psrc[it->second] = e;
          pscale[it->second] = sc;
        }
      }
    for (int v : csrc)
      if (v < 0) throw Error(SAP_ERR_CUDA, "update map: a band entry has no input entry");
    for (int v : psrc)
      if (v < 0) throw Error(SAP_ERR_CUDA, "update map: a coupling entry has no input entry");
    co_src.upload(csrc, st);
    co_scale.upload(cscale, st);
    cp_src.upload(psrc, st);
    cp_scale.upload(pscale, st);
  }

  // The numeric phase of the variable band: band (narrow) or blocks (wide)
  // from the diagonal-block entries, factors, spike tips, reduced system.
  void numeric_var() {
    if (ptype == SAP_PRECOND_NONE) return;
    auto t0 = Clock::now();
    if (use_wide(parts_maxK())) {
      wide_init(parts_maxK());
      wide->load_coo(co_row.get(), co_col.get(), co_val.get(), (long long)co_row.size());
      t_cpu_assemble += ms_since(t0);
      auto t2 = Clock::now();
      wide->factor(true);
      t_bandLU = ms_since(t2);
      if (spike) {
        coupling_dense();
        wide_couple(iface_h);
      }
      return;
    }
    wide.reset();
    B.alloc((size_t)boff_total);
    B.zero(st);
    {
      const long long m = (long long)co_row.size();
      k_band_from_coo_var<T><<<grid_for(m, 256, 148 * 32), 256, 0, st>>>(co_row.get(), co_col.get(), co_val.get(), m,
                                                                         parts_d.get(), partcol_d.get(), B.get());
      SAPB_LAUNCHED();
      SAPB_CUDA(cudaStreamSynchronize(st));
    }
    t_cpu_assemble += ms_since(t0);
    auto t2 = Clock::now();
    factor();
    t_bandLU = ms_since(t2);
    if (spike) {
      t2 = Clock::now();
      const size_t KK = (size_t)K * K;
      coupling_dense();
      iface_d.upload(iface_h, st);
      V.alloc(KK * (P - 1));
      W.alloc(KK * (P - 1));
      S.alloc(KK * (P - 1));
      int maxsz = 0;
      for (auto& d : parts_h) maxsz = std::max(maxsz, d.size);
      scratch.alloc((size_t)2 * (P - 1) * maxsz * K);
      if (K > 1024) throw Error(SAP_ERR_UNSUPPORTED, "coupling width above 1024 is not supported by the spike kernel");
      k_spikes_var<T><<<dim3(P - 1, 2), ((K + 31) / 32) * 32, 0, st>>>(parts_d.get(), B.get(), offd.get(), iface_d.get(),
                                                                   V.get(), W.get(), scratch.get(), (long long)maxsz, K);
      SAPB_LAUNCHED();
      SAPB_CUDA(cudaStreamSynchronize(st));
      scratch.release();
      t_assembly = ms_since(t2);
      t2 = Clock::now();
      k_reduced_factor<T><<<P - 1, 512, 0, st>>>(V.get(), W.get(), S.get(), K, o.safeFactorization ? 1 : 0);
      SAPB_LAUNCHED();
      SAPB_CUDA(cudaStreamSynchronize(st));
      t_fullLU = ms_since(t2);
    }
    build_sweeps();
  }

  void setup_from_band() {
    wide_active = false;
    ptype = o.precondType;
    spike = (ptype == SAP_PRECOND_SPIKE && P > 1);
    lu_ul = spike && o.factMethod == SAP_LU_UL;
    dscaled = false;
    if (ptype == SAP_PRECOND_NONE) return;
    init_parts_const();
    if (K == 0) return;
    if (tf32 && !reordered) {
      dscaled = true;
      dscale.alloc(n);
      k_diag_pow2<T><<<grid_for(n, 256), 256, 0, st>>>(B.get(), n, K, dscale.get());
      SAPB_LAUNCHED();
      k_band_scale<T><<<grid_for((long long)(2 * K + 1) * n, 256, 148 * 32), 256, 0, st>>>(B.get(), n, K,
                                                                                        dscale.get());
      SAPB_LAUNCHED();
    }
    auto t0 = Clock::now();
    if (spike) {
      offd.alloc((size_t)2 * (P - 1) * K * K);
      dim3 g(grid_for((long long)K * K, 256, 64), P - 1);
      k_extract_offdiag<T><<<g, 256, 0, st>>>(parts_d.get(), B.get(), offd.get(), K);
      SAPB_LAUNCHED();
    }
    SAPB_CUDA(cudaStreamSynchronize(st));
    t_offDiags = ms_since(t0);
    if (use_wide(K)) {
      wide_init(K);
      std::vector<long long> boff(P);
      std::vector<int> kp(P, K);
      for (int p = 0; p < P; p++) boff[p] = parts_h[p].boff;
      wide->load_band(B.get(), boff, kp);
      B.release();
      t0 = Clock::now();
      wide->factor(factor_boost());
      t_bandLU = ms_since(t0);
      if (spike) {
        std::vector<int> iface((size_t)(P - 1) * 2 * K);
        for (int i = 0; i < P - 1; i++) {
          const int s1 = parts_h[i + 1].start;
          for (int k = 0; k < K; k++) {
            iface[(size_t)i * 2 * K + k] = s1 - K + k;
            iface[(size_t)i * 2 * K + K + k] = s1 + k;
          }
        }
        wide_couple(iface);
      }
      return;
    }
    wide.reset();
    t0 = Clock::now();
    factor();
    SAPB_CUDA(cudaStreamSynchronize(st));
    t_bandLU = ms_since(t0);
    t0 = Clock::now();
    if (spike) {
      V.alloc((size_t)(P - 1) * K * K);
      W.alloc((size_t)(P - 1) * K * K);
      S.alloc((size_t)(P - 1) * K * K);
      if (lu_ul) {
        k_spikes_luul<T><<<dim3(P - 1, 2), ((K + 31) / 32) * 32, 0, st>>>(parts_d.get(), P, B.get(),
                                                                        B2.get() ? B2.get() : B.get(), offd.get(),
                                                                        V.get(), W.get(), K);
        SAPB_LAUNCHED();
      } else {
        int maxsz = 0;
        for (auto& p : parts_h) maxsz = std::max(maxsz, p.size);
        scratch.alloc((size_t)(P - 1) * K * maxsz);
        k_spikes_luonly<T><<<dim3(P - 1, 2), ((K + 31) / 32) * 32, 0, st>>>(parts_d.get(), B.get(), offd.get(),
                                                                          V.get(), W.get(), scratch.get(),
                                                                          (long long)maxsz, K);
        SAPB_LAUNCHED();
      }
      SAPB_CUDA(cudaStreamSynchronize(st));
      B2.release();
      scratch.release();
      t_assembly = ms_since(t0);
      t0 = Clock::now();
      k_reduced_factor<T><<<P - 1, 512, 0, st>>>(V.get(), W.get(), S.get(), K, o.safeFactorization ? 1 : 0);
      SAPB_LAUNCHED();
      SAPB_CUDA(cudaStreamSynchronize(st));
      t_fullLU = ms_since(t0);
    }
    build_sweeps();
  }

  // partBandedLU / partBlockedBandedUL (sap/precond.h:3882-3983, 4336-4418, 4780-4846).
  void factor() {
    std::vector<FactorJob> jobs;
    const bool boost = factor_boost();
    // the variable-band kernels always boost (partBlockedBandedLU_var, precond.h:4546-4631)
    if (var_band || !spike) {
      for (const auto& d : parts_h) jobs.push_back(FactorJob{d.start, d.start + d.size, d.K, 0, 0, 0, d.boff});
    } else {
      int nlu = lu_ul ? P - 1 : P;
      for (int p = 0; p < nlu; p++) {
        const auto& d = parts_h[p];
        jobs.push_back(FactorJob{d.start, d.start + d.size, d.K, 0, 0, 0, d.boff});
      }
      if (lu_ul) {
        if (P > 2) {
          B2.alloc(B.size());
          SAPB_CUDA(cudaMemcpyAsync(B2.get(), B.get(), B.size() * sizeof(T), cudaMemcpyDeviceToDevice, st));
        }
        for (int p = 1; p < P; p++) {
          const auto& d = parts_h[p];
          int target = (p == P - 1) ? 0 : 1;
          jobs.push_back(FactorJob{d.start, d.start + d.size, d.K, 1, target, 0, d.boff});
        }
      }
    }
    DBuf<FactorJob> jobs_d;
    jobs_d.upload(jobs, st);
    flag.alloc(1);  // a zero pivot seen
    flag.zero(st);
    const int Kmax = parts_maxK();
    int G = std::max(1, std::min(Kmax, 512 / std::max(Kmax, 1)));
    int NT = ((Kmax * G + 31) / 32) * 32;
    NT = std::max(NT, 64);
    constexpr int D = 8;
    size_t smem = ((size_t)(Kmax + 1 + D) * (2 * Kmax + 1) + (Kmax + 1 + D)) * sizeof(T);
    constexpr int NB = 8;
    const char* fk = std::getenv("SAPB_FACTOR_KERNEL");
    const bool ring_only = fk && std::string(fk) == "ring";
    const int R = (Kmax + NB + 31) / 32;
    int maxrows = 0;
    for (const auto& jb : jobs) maxrows = std::max(maxrows, jb.e - jb.s);
    auto postdiv = [&]() {
      SAPB_LAUNCHED();
      k_factor_postdiv<T><<<dim3(grid_for((long long)maxrows * Kmax, 256, 1024), (int)jobs.size()), 256, 0, st>>>(
          jobs_d.get(), B.get(), B2.get());
    };
    auto panel_smem = [&](int dpf) { return (size_t)(Kmax + NB * (1 + dpf)) * (2 * Kmax + 1) * sizeof(T); };
    if (!ring_only && R <= 4 && panel_smem(1) <= 227 * 1024) {
      const int dpf = panel_smem(2) <= 227 * 1024 ? 2 : 1;
      const size_t psm = panel_smem(dpf);
      const int nt = 32 * std::min(16, std::max(2, (Kmax + 3) / 4));  // four trailing columns per warp
      auto launch = [&](auto kern) {
        SAPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
        kern<<<(int)jobs.size(), nt, psm, st>>>(jobs_d.get(), B.get(), B2.get(), boost ? 1 : 0, flag.get(), dpf);
      };
      SAPB_PROF("factor", st);  // the factor kernel and its post-divide pass
      switch (R) {
        case 1: launch(k_factor_panel<T, NB, 1>); break;
        case 2: launch(k_factor_panel<T, NB, 2>); break;
        case 3: launch(k_factor_panel<T, NB, 3>); break;
        default: launch(k_factor_panel<T, NB, 4>); break;
      }
      postdiv();
    } else if (smem <= 200 * 1024) {
      SAPB_CUDA(cudaFuncSetAttribute(k_factor_smem<T, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      SAPB_PROF("factor", st);
      k_factor_smem<T, D><<<(int)jobs.size(), NT, smem, st>>>(jobs_d.get(), B.get(), B2.get(), boost ? 1 : 0,
                                                             flag.get(), G);
    } else {
      SAPB_PROF("factor", st);
      k_factor_global<T><<<(int)jobs.size(), NT, 0, st>>>(jobs_d.get(), B.get(), B2.get(), boost ? 1 : 0, flag.get(), G);
    }
    SAPB_LAUNCHED();
    int hflag = 0;
    SAPB_CUDA(cudaMemcpyAsync(&hflag, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    SAPB_CUDA(cudaStreamSynchronize(st));
    if (hflag && !o.safeFactorization && !boost)
      throw Error(SAP_ZERO_PIVOTING, "Found a pivot equal to zero (partBandedLU).");
  }

  void build_sweeps() {
    int maxK = parts_maxK();
    if (maxK > 1024) throw Error(SAP_ERR_UNSUPPORTED, "half-bandwidth above 1024 is not supported by the sweep kernels");
    chunks_h.clear();
    std::vector<long long> koff, toff;
    std::vector<int> first1, first2, pc0, pnc;
    long long ko = 0, to = 0;
    maxChunk = 0;
    for (int p = 0; p < (int)parts_h.size(); p++) {
      const auto& d = parts_h[p];
      int Kp = d.K;
      int m = std::min(4096, std::max(256, 8 * Kp));
      int nc = std::max(1, d.size / m);
      pc0.push_back((int)chunks_h.size());
      pnc.push_back(nc);
      int base = d.size / nc, rem = d.size % nc, a = d.start;
      for (int c = 0; c < nc; c++) {
        int len = base + (c < rem ? 1 : 0);
        chunks_h.push_back(ChunkDev{p, a, a + len, 0});
        maxChunk = std::max(maxChunk, len);
        koff.push_back(ko);
        toff.push_back(to);
        ko += Kp;
        to += (long long)Kp * Kp;
        bool down1 = !d.ul;
        first1.push_back(down1 ? (c == 0) : (c == nc - 1));
        first2.push_back(down1 ? (c == nc - 1) : (c == 0));
        a += len;
      }
    }
    chunks_d.upload(chunks_h, st);
    koff_d.upload(koff, st);
    toff_d.upload(toff, st);
    first1_d.upload(first1, st);
    first2_d.upload(first2, st);
    pchunk0_d.upload(pc0, st);
    pnchunk_d.upload(pnc, st);
    T1.alloc(std::max<long long>(to, 1));
    T2.alloc(std::max<long long>(to, 1));
    tails1.alloc(std::max<long long>(ko, 1));
    tails2.alloc(std::max<long long>(ko, 1));
    carry1.alloc(std::max<long long>(ko, 1));
    carry2.alloc(std::max<long long>(ko, 1));
    F.alloc(n);
    Gv.alloc(n);
    Y.alloc(n);
    sweepThreads = std::max(32, ((maxK + 31) / 32) * 32);
    scanG = std::max(1, std::min(maxK, 512 / std::max(1, maxK)));
    const int nch = (int)chunks_h.size();
    const int tthreads = sweepThreads;
    size_t tsmem = (size_t)maxK * tthreads * sizeof(T);
    DBuf<T> gring;
    auto t0 = Clock::now();
    if (tsmem > 200 * 1024) {
      gring.alloc((size_t)nch * maxK * tthreads);
      tsmem = 0;
    } else {
      SAPB_CUDA(cudaFuncSetAttribute(k_transfer<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(tsmem, 1024)));
    }
    SAPB_PROF("transfer", st);
    k_transfer<T><<<nch, tthreads, tsmem, st>>>(parts_d.get(), chunks_d.get(), toff_d.get(), B.get(), T1.get(), 1, gring.get(), first1_d.get());
    SAPB_LAUNCHED();
    k_transfer<T><<<nch, tthreads, tsmem, st>>>(parts_d.get(), chunks_d.get(), toff_d.get(), B.get(), T2.get(), 2, gring.get(), first2_d.get());
    SAPB_LAUNCHED();
    size_t s1 = (size_t)(maxK + maxChunk) * sizeof(T);
    if (2 * s1 > 220 * 1024) throw Error(SAP_ERR_UNSUPPORTED, "sweep chunk does not fit in shared memory");
    SAPB_CUDA(cudaFuncSetAttribute(k_pass2<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * s1)));
    SAPB_CUDA(cudaFuncSetAttribute(k_pass1<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1));
    SAPB_CUDA(cudaFuncSetAttribute(k_pass3<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1));
    SAPB_CUDA(cudaStreamSynchronize(st));
    t_assembly += ms_since(t0);
  }

  // One partitioned sweep pair: out = D^-1 rhs, rhs = vin (FP64) or F.
  void sweep_pair(const double* vin, double* zout, T* gout) {
    const int nch = (int)chunks_h.size();
    const int maxK = parts_maxK();
    const size_t s1 = (size_t)(maxK + maxChunk) * sizeof(T);
    const int NT = sweepThreads;
    const int scanNT = ((maxK * scanG + 31) / 32) * 32;
    const size_t ssm = (size_t)(maxK + scanG * maxK) * sizeof(T);
    {
      SAPB_PROF("pass1", st);
      k_pass1<T, 16><<<nch, NT, s1, st>>>(parts_d.get(), chunks_d.get(), koff_d.get(), B.get(), vin, F.get(), tails1.get(),
                                          reordered ? gin_d.get() : nullptr, in_scale());
      SAPB_LAUNCHED();
    }
    {
      SAPB_PROF("scan", st);
      k_scan<T><<<(int)parts_h.size(), scanNT, ssm, st>>>(parts_d.get(), pchunk0_d.get(), pnchunk_d.get(), koff_d.get(),
                                                          toff_d.get(), T1.get(), tails1.get(), carry1.get(), 1, scanG);
      SAPB_LAUNCHED();
    }
    {
      SAPB_PROF("pass2", st);
      k_pass2<T, 16><<<nch, NT, 2 * s1, st>>>(parts_d.get(), chunks_d.get(), first1_d.get(), koff_d.get(), B.get(),
                                              F.get(), carry1.get(), Y.get(), tails2.get());
      SAPB_LAUNCHED();
    }
    {
      SAPB_PROF("scan", st);
      k_scan<T><<<(int)parts_h.size(), scanNT, ssm, st>>>(parts_d.get(), pchunk0_d.get(), pnchunk_d.get(), koff_d.get(),
                                                          toff_d.get(), T2.get(), tails2.get(), carry2.get(), 2, scanG);
      SAPB_LAUNCHED();
    }
    {
      SAPB_PROF("pass3", st);
      k_pass3<T, 16><<<nch, NT, s1, st>>>(parts_d.get(), chunks_d.get(), first2_d.get(), koff_d.get(), B.get(), Y.get(),
                                          carry2.get(), zout, gout, reordered ? sout_d.get() : nullptr,
                                          out_scale());
      SAPB_LAUNCHED();
    }
  }

  // Precond::operator() + solve + getSRev (sap/precond.h:1370-1528) in the
  // band's row order.
  void check_device() override {
    if (wide) wide->check_device();
  }

  void apply_band(const double* v, double* z) override {
    if (ptype == SAP_PRECOND_NONE) {
      SAPB_CUDA(cudaMemcpyAsync(z, v, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
      return;
    }
    if (K == 0) {
      if (reordered) throw Error(SAP_ERR_UNSUPPORTED, "a diagonal matrix after reordering is not supported");
      k_diag_apply<T><<<grid_for(n, 256), 256, 0, st>>>(B.get(), v, z, n);
      SAPB_LAUNCHED();
      return;
    }
    if (wide_active) {
      wide->apply(v, z, reordered ? gin_d.get() : nullptr, in_scale(), reordered ? sout_d.get() : nullptr,
                  out_scale());
      return;
    }
    if (spike) {
      sweep_pair(v, nullptr, Gv.get());
      {
      SAPB_PROF("reduced_apply", st);
      k_reduced_apply<T><<<P - 1, ((K + 31) / 32) * 32, 3 * K * sizeof(T), st>>>(parts_d.get(), V.get(), W.get(), S.get(),
                                                                            offd.get(), Gv.get(), F.get(), K,
                                                                            var_band ? iface_d.get() : nullptr);
      SAPB_LAUNCHED();
      }
      sweep_pair(nullptr, z, nullptr);
    } else {
      sweep_pair(v, z, nullptr);
    }
  }
};

// ---------------------------------------------------------------------------
// BiCGStabLMonitor (sap/monitor.h:154-339).
struct Monitor {
  int maxIt = 100, maxm = 8, stag = 0, more = 0, maxStag = 3;
  double relTol = 1e-6, absTol = 0, rhsNorm = 0, rNorm = std::numeric_limits<double>::max();
  float it = 0;
  int code = 0;
  std::string msg;
  void init(double rhs) { rhsNorm = rhs; it = 0; code = 0; msg = ""; stag = 0; more = 0; }
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

// ---------------------------------------------------------------------------
class Solver {
 public:
  sap_options opts{};
  int P_req = 1;
  int prec_dtype = SAP_PREC_FLOAT;
  cudaStream_t st = nullptr;
  std::unique_ptr<PrecBase> pcp;
  PrecBase& pc() { return *pcp; }
  Monitor mon;
  sap_stats stats{};
  bool setup_done = false;
  int n = 0;
  long long nnz = 0;
  // Krylov workspace
  DBuf<double> dots_part, dots_out;
  DBuf<unsigned int> dots_ctr;
  // classical Gram-Schmidt of flexible GMRES: basis pointers, partials,
  // counters, the two passes' coefficients
  DBuf<const double*> gs_v;
  DBuf<double> gs_part, gs_h;
  DBuf<unsigned int> gs_ctr;
  double* pinned = nullptr;
  DBuf<double> bvec, xvec;
  // persistent Krylov vectors (allocated at the first solve of size n)
  std::vector<DBuf<double>> ws;
  double* wsv(int i) {
    if ((int)ws.size() <= i) ws.resize(i + 1);
    ws[i].alloc(n);
    return ws[i].get();
  }

  Solver(int P, const sap_options& o, int dtype) : opts(o), P_req(P), prec_dtype(dtype) {
    SAPB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (dtype == SAP_PREC_DOUBLE) pcp = std::make_unique<PrecondT<double>>();
    else pcp = std::make_unique<PrecondT<float>>();
    pcp->tf32 = dtype == SAP_PREC_TF32 || dtype == SAP_PREC_TF32_F16;
    pcp->h16 = dtype == SAP_PREC_TF32_F16;
    pcp->o = o;
    pcp->P_req = P;
    pcp->st = st;
    mon.maxIt = o.maxNumIterations;
    mon.relTol = o.relTol;
    mon.absTol = o.absTol;
    dots_part.alloc(4 * kDotBlocks);
    dots_out.alloc(4);
    dots_ctr.alloc(1);
    dots_ctr.zero(st);
    SAPB_CUDA(cudaMallocHost(&pinned, (2 * kMaxBasis + 8) * sizeof(double)));
    init_stats();
  }
  ~Solver() {
    if (pinned) cudaFreeHost(pinned);
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  }
  void init_stats() {
    std::memset(&stats, 0, sizeof(stats));
    stats.rhsNorm = stats.residualNorm = stats.relResidualNorm = std::numeric_limits<double>::max();
  }

  // -- BLAS-1 on the solver stream ------------------------------------------
  void axpby(const double* x, const double* y, double* z, double a, double b) {
    k_axpby<<<grid_for(n, 256), 256, 0, st>>>(n, a, x, b, y, z);
    SAPB_LAUNCHED();
  }
  void axpy(const double* x, double* y, double a) {
    k_axpy<<<grid_for(n, 256), 256, 0, st>>>(n, a, x, y);
    SAPB_LAUNCHED();
  }
  void copy(const double* x, double* y) {
    SAPB_CUDA(cudaMemcpyAsync(y, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  // up to four dot products, returned on the host
  void dots(int nq, const double* const* xs, const double* const* ys, double* out) {
    DotArgs a{};
    a.nq = nq;
    for (int q = 0; q < nq; q++) { a.x[q] = xs[q]; a.y[q] = ys[q]; }
    {
      SAPB_PROF("dots", st);
      k_dots<<<kDotBlocks, kDotThreads, 0, st>>>(n, a, dots_part.get(), dots_ctr.get(), dots_out.get());
      SAPB_LAUNCHED();
    }
    SAPB_CUDA(cudaMemcpyAsync(pinned, dots_out.get(), nq * sizeof(double), cudaMemcpyDeviceToHost, st));
    SAPB_CUDA(cudaStreamSynchronize(st));
    for (int q = 0; q < nq; q++) out[q] = pinned[q];
  }
  double dot(const double* x, const double* y) {
    double r;
    dots(1, &x, &y, &r);
    return r;
  }
  // ||w||^2 into dots_out[0] on the device, no synchronisation
  void sqnorm_dev(const double* w) {
    DotArgs a{};
    a.nq = 1;
    a.x[0] = w;
    a.y[0] = w;
    SAPB_PROF("dots", st);
    k_dots<<<kDotBlocks, kDotThreads, 0, st>>>(n, a, dots_part.get(), dots_ctr.get(), dots_out.get());
    SAPB_LAUNCHED();
  }
  // one classical Gram-Schmidt pass against basis vectors 0..m-1 (device
  // pointer array vs): h = V^T w, w -= V h
  void cgs_pass(int m, const double* const* vs, double* w, double* h) {
    {
      SAPB_PROF("dots", st);
      k_mdot<<<dim3(kMdotBlocks, m), kMdotThreads, 0, st>>>(n, vs, w, gs_part.get(), gs_ctr.get(), h);
      SAPB_LAUNCHED();
    }
    k_maxpy<<<grid_for(n, 256), 256, 0, st>>>(n, m, vs, h, w);
    SAPB_LAUNCHED();
  }
  double nrm2(const double* x) { return std::sqrt(dot(x, x)); }
  // y += a x and ||y|| from one pass (the values of axpy then nrm2)
  double axpy_nrm2(const double* x, double* y, double a) {
    {
      SAPB_PROF("dots", st);
      k_axpy_sqnorm<<<kDotBlocks, kDotThreads, 0, st>>>(n, a, x, y, dots_part.get(), dots_ctr.get(), dots_out.get());
      SAPB_LAUNCHED();
    }
    SAPB_CUDA(cudaMemcpyAsync(pinned, dots_out.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    SAPB_CUDA(cudaStreamSynchronize(st));
    return std::sqrt(pinned[0]);
  }

  // bicgstabl<..., L> (sap/bicgstab2.h:32-360)
  void bicgstabl(const Spmv& A, double* x, const double* b, int L);

  // Flexible GMRES(m) (Saad, SIAM J. Sci. Comput. 14 (1993) 461-469):
  // right preconditioning with the preconditioned directions z_j kept, so
  // the preconditioner may vary between applies; FP64 Arnoldi with classical
  // Gram-Schmidt applied twice (CGS2: Giraud, Langou, Rozloznik, Comput.
  // Math. Appl. 50 (2005) 1069-1075 -- orthogonal to working precision like
  // modified Gram-Schmidt), each pass one multi-dot and one multi-axpy launch
  // with the coefficients kept on the device, the norm and normalisation on
  // the device, and one host synchronisation per Arnoldi step; Givens
  // rotations for the least-squares residual, the true residual b - A x
  // checked after every cycle.  Monitor: 1 converged, -1 iteration budget,
  // -2 NaN, -3 a cycle that did not lower the residual.
  void fgmres(const Spmv& A, double* x, const double* b, int m) {
    if (m + 1 > kMaxBasis) throw Error(SAP_ERR_UNSUPPORTED, "FGMRES restart length above the Gram-Schmidt limit");
    const double tol = mon.tol();
    double* r = wsv(39);
    std::vector<double*> Vb(m + 1), Zb(m);
    for (int i = 0; i <= m; i++) Vb[i] = wsv(40 + i);
    for (int i = 0; i < m; i++) Zb[i] = wsv(41 + m + i);
    std::vector<const double*> vptr(Vb.begin(), Vb.end());
    gs_v.upload(vptr, st);
    gs_part.ensure((size_t)kMdotBlocks * kMaxBasis);
    gs_h.ensure(2 * kMaxBasis);
    if (gs_ctr.size() < (size_t)kMaxBasis) {
      gs_ctr.alloc(kMaxBasis);
      gs_ctr.zero(st);
    }
    double* h1 = gs_h.get();
    double* h2 = gs_h.get() + kMaxBasis;
    std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m, 0.0), sn(m, 0.0), g(m + 1, 0.0);
    auto h = [&](int i, int j) -> double& { return H[(size_t)i * m + j]; };
    auto residual = [&]() {
      A.apply(x, r, st);
      axpby(b, r, r, 1.0, -1.0);
      return nrm2(r);
    };
    double beta = residual();
    int total = 0;
    while (true) {
      mon.rNorm = beta;
      if (std::isnan(beta)) { mon.stop(-2, "Residual norm is NaN"); break; }
      if (beta <= tol) { mon.stop(1, "Converged"); break; }
      if (total >= mon.maxIt) { mon.stop(-1, "Maximum number of iterations was reached"); break; }
      axpby(r, r, Vb[0], 1.0 / beta, 0.0);
      std::fill(g.begin(), g.end(), 0.0);
      g[0] = beta;
      int j = 0;
      bool nan = false;
      while (j < m && total < mon.maxIt) {
        pcp->apply(Vb[j], Zb[j]);
        A.apply(Zb[j], Vb[j + 1], st);
        cgs_pass(j + 1, gs_v.get(), Vb[j + 1], h1);
        cgs_pass(j + 1, gs_v.get(), Vb[j + 1], h2);
        sqnorm_dev(Vb[j + 1]);
        k_scale_inv_norm<<<grid_for(n, 256), 256, 0, st>>>(n, Vb[j + 1], dots_out.get());
        SAPB_LAUNCHED();
        SAPB_CUDA(cudaMemcpyAsync(pinned, gs_h.get(), (size_t)(j + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
        SAPB_CUDA(cudaMemcpyAsync(pinned + kMaxBasis, h2, (size_t)(j + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                                  st));
        SAPB_CUDA(cudaMemcpyAsync(pinned + 2 * kMaxBasis, dots_out.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
        SAPB_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i <= j; i++) h(i, j) = pinned[i] + pinned[kMaxBasis + i];
        const double hn = std::sqrt(pinned[2 * kMaxBasis]);
        h(j + 1, j) = hn;
        for (int i = 0; i < j; i++) {  // previous rotations on column j
          const double a = h(i, j), c = h(i + 1, j);
          h(i, j) = cs[i] * a + sn[i] * c;
          h(i + 1, j) = -sn[i] * a + cs[i] * c;
        }
        const double a = h(j, j), c = h(j + 1, j);
        const double rho = std::hypot(a, c);
        cs[j] = rho > 0 ? a / rho : 1.0;
        sn[j] = rho > 0 ? c / rho : 0.0;
        h(j, j) = rho;
        h(j + 1, j) = 0.0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        j++;
        total++;
        mon.it = (float)total;
        const double est = std::fabs(g[j]);
        if (std::isnan(est)) { nan = true; break; }
        if (est <= tol || hn == 0) break;
      }
      // y = R^-1 g, x += Z y
      std::vector<double> y(j, 0.0);
      for (int i = j - 1; i >= 0; i--) {
        double s = g[i];
        for (int k = i + 1; k < j; k++) s -= h(i, k) * y[k];
        y[i] = h(i, i) != 0 ? s / h(i, i) : 0.0;
      }
      for (int i = 0; i < j; i++) axpy(Zb[i], x, y[i]);
      const double bnew = residual();
      if (nan || std::isnan(bnew)) { mon.rNorm = bnew; mon.stop(-2, "Residual norm is NaN"); break; }
      const bool progress = bnew < beta;
      beta = bnew;
      if (!progress && beta > tol) { mon.rNorm = beta; mon.stop(-3, "Stagnation encountered"); break; }
    }
    SAPB_CUDA(cudaStreamSynchronize(st));
  }

  // Monitor::finished (sap/monitor.h:134-149): the default monitor of the
  // BiCGStab and MINRES drivers.
  bool finished_default(double r) {
    mon.rNorm = r;
    if (mon.code != 0) return true;
    if (std::isnan(r)) mon.stop(-2, "Residual norm is NaN");
    else if (r <= mon.tol()) mon.stop(1, "Converged");
    else if (mon.it > mon.maxIt) mon.stop(-1, "Maximum number of iterations was reached");
    return mon.code != 0;
  }
  void axpbypcz(const double* x, const double* y, const double* z, double* out, double a, double b, double c) {
    k_axpbypcz<<<grid_for(n, 256), 256, 0, st>>>(n, a, x, b, y, c, z, out);
    SAPB_LAUNCHED();
  }

  // sap::bicgstab (sap/bicgstab.h:50-155)
  void bicgstab_classic(const Spmv& A, double* x, const double* b) {
    double *y = wsv(70), *p = wsv(71), *r = wsv(72), *rs = wsv(73), *s = wsv(74), *Mp = wsv(75), *AMp = wsv(76),
           *Ms = wsv(77), *AMs = wsv(78);
    A.apply(x, y, st);
    axpby(b, y, r, 1.0, -1.0);
    copy(r, p);
    copy(r, rs);
    double rr_old = dot(rs, r);
    while (!finished_default(nrm2(r))) {
      if (rr_old == 0) { mon.stop(-10, "r_r_star is zero"); break; }
      pcp->apply(p, Mp);
      A.apply(Mp, AMp, st);
      const double t1 = dot(rs, AMp);
      if (t1 == 0) { mon.stop(-11, "r_star * AMp is zero"); break; }
      const double alpha = rr_old / t1;
      axpby(r, AMp, s, 1.0, -alpha);
      if (finished_default(nrm2(s))) {
        axpby(x, Mp, x, 1.0, alpha);
        break;
      }
      pcp->apply(s, Ms);
      A.apply(Ms, AMs, st);
      const double t2 = dot(AMs, AMs);
      if (t2 == 0) { mon.stop(-12, "AMs * AMs is zero"); break; }
      const double omega = dot(AMs, s) / t2;
      axpbypcz(x, Mp, Ms, x, 1.0, alpha, omega);
      axpby(s, AMs, r, 1.0, -omega);
      const double rr_new = dot(rs, r);
      const double beta = (rr_new / rr_old) * (alpha / omega);
      rr_old = rr_new;
      axpbypcz(r, p, AMp, p, 1.0, beta, -beta * omega);
      mon.it += 1.f;
    }
    SAPB_CUDA(cudaStreamSynchronize(st));
  }

  // sap::minres (sap/minres.h:40-195): preconditioned Lanczos with Givens
  // rotations, stop codes 10-13 and -10 as in the reference.
  void minres(const Spmv& A, double* x, const double* b) {
    const double eps = std::numeric_limits<double>::epsilon();
    auto count = [&]() { return (size_t)(mon.it + 0.5f); };
    double *y = wsv(80), *r1 = wsv(81), *v = wsv(82), *w = wsv(83), *w1 = wsv(84), *w2 = wsv(85), *r2 = wsv(86);
    A.apply(x, r1, st);
    axpby(b, r1, r1, 1.0, -1.0);
    pcp->apply(r1, y);
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
    for (double* q : {w, w1, w2}) SAPB_CUDA(cudaMemsetAsync(q, 0, (size_t)n * sizeof(double), st));
    copy(r1, r2);
    while (!finished_default(phibar)) {
      const double s = 1 / beta;
      axpby(y, y, v, s, 0.0);
      A.apply(v, y, st);
      if (count() > 0) axpby(y, r1, y, 1.0, -beta / oldb);
      alpha = dot(v, y);
      axpby(y, r2, y, 1.0, -alpha / beta);
      copy(r2, r1);
      copy(y, r2);
      pcp->apply(r2, y);
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
      copy(w2, w1);
      copy(w, w2);
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
    SAPB_CUDA(cudaStreamSynchronize(st));
  }

  // The Krylov method of the options: L > 0 BiCGStab(L), L == 0 flexible
  // GMRES(50), L == -1 sap::bicgstab, L == -2 sap::minres.
  void krylov(const Spmv& A, double* x, const double* b, int L) {
    if (L > 0) bicgstabl(A, x, b, L);
    else if (L == 0) fgmres(A, x, b, 50);
    else if (L == -1) bicgstab_classic(A, x, b);
    else minres(A, x, b);
  }

  // FP64 iterative refinement around bicgstabl (options.refinementSweeps):
  // every sweep solves A d = r for the true residual r = b - A x to the
  // global tolerance (or until the inner monitor stops), then x += d.  The
  // monitor reports the final true residual and the total iteration count.
  void refine(const Spmv& A, double* x, const double* b, int L, int sweeps) {
    // slots 30, 31: beyond bicgstabl's (2L+2+10 <= 16 for L <= 2)
    struct Vec {
      double* p;
      double* get() const { return p; }
    } r{wsv(30)}, d{wsv(31)};
    const double bn = mon.rhsNorm;
    const double tol = opts.absTol + opts.relTol * bn;
    auto residual = [&]() {
      A.apply(x, r.get(), st);
      axpby(b, r.get(), r.get(), 1.0, -1.0);
      return nrm2(r.get());
    };
    double rn = residual();
    float total = 0;
    int code = 0;
    std::string msg;
    for (int sw = 0; sw < sweeps; sw++) {
      if (rn <= tol) break;
      const float left = (float)opts.maxNumIterations - total;
      if (left <= 0) { code = -1; msg = "Maximum number of iterations was reached"; break; }
      SAPB_CUDA(cudaMemsetAsync(d.p, 0, (size_t)n * sizeof(double), st));
      mon.init(rn);
      mon.relTol = tol / rn;
      mon.absTol = 0;
      mon.maxIt = (int)std::ceil(left);
      krylov(A, d.get(), r.get(), L);
      total += mon.it;
      code = mon.code;
      msg = mon.msg;
      axpy(d.get(), x, 1.0);
      const double rnew = residual();
      const bool progress = rnew < rn;
      rn = rnew;
      if (!progress) break;
    }
    mon.relTol = opts.relTol;
    mon.absTol = opts.absTol;
    mon.maxIt = opts.maxNumIterations;
    mon.rhsNorm = bn;
    mon.rNorm = rn;
    mon.it = total;
    if (std::isnan(rn)) { code = -2; msg = "Residual norm is NaN"; }
    else if (rn <= tol) { code = 1; msg = "Converged"; }
    else if (code > 0) { code = -3; msg = "Stagnation encountered"; }
    mon.code = code;
    mon.msg = msg;
    SAPB_CUDA(cudaStreamSynchronize(st));
  }
};

void Solver::bicgstabl(const Spmv& A, double* x, const double* b, int L) {
  const double eps = 1e-20;
  double rho0 = 1, alpha = 0, omega = 1, rho1;
  // workspace slots 0..2L+1: rr, uu; then the named vectors
  struct Vec {
    double* p;
    double* get() const { return p; }
  };
  std::vector<Vec> rr(L + 1), uu(L + 1);
  for (int k = 0; k <= L; k++) {
    rr[k].p = wsv(k);
    uu[k].p = wsv(L + 1 + k);
    SAPB_CUDA(cudaMemsetAsync(rr[k].p, 0, (size_t)n * sizeof(double), st));
    SAPB_CUDA(cudaMemsetAsync(uu[k].p, 0, (size_t)n * sizeof(double), st));
  }
  const int w0 = 2 * L + 2;
  Vec r0{wsv(w0)}, xx{wsv(w0 + 1)}, Pv{wsv(w0 + 2)}, x_min{wsv(w0 + 3)}, Pxx{wsv(w0 + 4)}, APxx{wsv(w0 + 5)};
  SAPB_CUDA(cudaMemsetAsync(x_min.p, 0, (size_t)n * sizeof(double), st));
  std::vector<std::vector<double>> tao(L + 1, std::vector<double>(L + 1, 0.0));
  std::vector<double> gamma(L + 2), gp(L + 2), gpp(L + 2), sigma(L + 2);
  auto Pm = [&](const double* in, double* out) { pcp->apply(in, out); };
  auto Am = [&](const double* in, double* out) { A.apply(in, out, st); };

  // r0 <- b - A x ; r <- r0 ; uu0 <- 0 ; xx <- x ; rr0 <- r
  Am(x, r0.get());
  axpby(b, r0.get(), r0.get(), 1.0, -1.0);
  copy(x, xx.get());
  copy(r0.get(), rr[0].get());
  double r_norm_min = nrm2(rr[0].get()), r_norm = r_norm_min, r_norm_act = r_norm;
  auto recheck = [&]() {
    Pm(xx.get(), Pxx.get());
    Am(Pxx.get(), APxx.get());
    axpby(b, APxx.get(), rr[0].get(), 1.0, -1.0);
    r_norm_act = nrm2(rr[0].get());
  };
  auto stag_check = [&](double coef, const double* v) {
    const double* xs[2] = {v, xx.get()};
    double d[2];
    dots(2, xs, xs, d);
    if (std::fabs(coef) * std::sqrt(d[0]) < eps * std::sqrt(d[1])) mon.stag++;
    else mon.stag = 0;
  };
  while (true) {
    rho0 = -omega * rho0;
    mon.it += 0.25f;
    for (int j = 0; j < L; j++) {
      rho1 = dot(rr[j].get(), r0.get());
      if (rho0 == 0) { mon.stop(-10, "rho0 is zero"); break; }
      double beta = alpha * rho1 / rho0;
      rho0 = rho1;
      for (int i = 0; i <= j; i++) axpby(rr[i].get(), uu[i].get(), uu[i].get(), 1.0, -beta);
      Pm(uu[j].get(), Pv.get());
      Am(Pv.get(), uu[j + 1].get());
      double gam = dot(uu[j + 1].get(), r0.get());
      if (gam == 0) { mon.stop(-11, "gamma is zero"); break; }
      alpha = rho0 / gam;
      r_norm_act = r_norm = axpy_nrm2(uu[1].get(), rr[0].get(), -alpha);  // rr_0 -= alpha uu_1, ||rr_0||
      for (int i = 1; i <= j; i++) axpy(uu[i + 1].get(), rr[i].get(), -alpha);
      Pm(rr[j].get(), Pv.get());
      Am(Pv.get(), rr[j + 1].get());
      stag_check(alpha, uu[0].get());
      axpy(uu[0].get(), xx.get(), alpha);
      if (mon.needCheck(r_norm)) {
        recheck();
        if (mon.finished(r_norm_act)) break;
      }
      if (r_norm_act < r_norm_min) { r_norm_min = r_norm_act; copy(xx.get(), x_min.get()); }
      if (mon.finished()) break;
    }
    if (mon.finished()) break;
    for (int j = 1; j <= L; j++) {
      for (int i = 1; i < j; i++) {
        tao[i][j] = dot(rr[j].get(), rr[i].get()) / sigma[i];
        axpy(rr[i].get(), rr[j].get(), -tao[i][j]);
      }
      const double* xs[2] = {rr[j].get(), rr[j].get()};
      const double* ys[2] = {rr[j].get(), rr[0].get()};
      double d[2];
      dots(2, xs, ys, d);
      sigma[j] = d[0];
      if (sigma[j] == 0) { mon.stop(-12, "a sigma value is zero"); break; }
      gp[j] = d[1] / sigma[j];
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
    stag_check(gamma[1], rr[0].get());
    axpy(rr[0].get(), xx.get(), gamma[1]);
    r_norm_act = r_norm = axpy_nrm2(rr[L].get(), rr[0].get(), -gp[L]);
    axpy(uu[L].get(), uu[0].get(), -gamma[L]);
    mon.it += 0.25f;
    if (mon.needCheck(r_norm)) {
      recheck();
      if (mon.finished(r_norm_act)) break;
    }
    if (r_norm_act < r_norm_min) { r_norm_min = r_norm_act; copy(xx.get(), x_min.get()); }
    if (mon.finished()) break;
    mon.it += 0.25f;
    for (int j = 1; j < L; j++) {
      axpy(uu[j].get(), uu[0].get(), -gamma[j]);
      stag_check(gpp[j], rr[j].get());
      axpy(rr[j].get(), xx.get(), gpp[j]);
      r_norm_act = r_norm = axpy_nrm2(rr[j].get(), rr[0].get(), -gp[j]);
      if (mon.needCheck(r_norm)) {
        recheck();
        if (mon.finished(r_norm_act)) break;
      }
      if (r_norm_act < r_norm_min) { r_norm_min = r_norm_act; copy(xx.get(), x_min.get()); }
      if (mon.finished()) break;
    }
    if (mon.finished()) break;
    mon.it += 0.25f;
  }
  if (mon.code > 0) {
    Pm(xx.get(), x);
  } else {
    Vec Pxmin{wsv(w0 + 6)}, APxmin{wsv(w0 + 7)}, rc{wsv(w0 + 8)}, rcm{wsv(w0 + 9)};
    Pm(xx.get(), Pxx.get());
    Am(Pxx.get(), APxx.get());
    axpby(b, APxx.get(), rc.get(), 1.0, -1.0);
    Pm(x_min.get(), Pxmin.get());
    Am(Pxmin.get(), APxmin.get());
    axpby(b, APxmin.get(), rcm.get(), 1.0, -1.0);
    double a = nrm2(rc.get()), c = nrm2(rcm.get());
    if (a < c) { copy(Pxx.get(), x); mon.rNorm = a; }
    else { copy(Pxmin.get(), x); mon.rNorm = c; }
  }
  SAPB_CUDA(cudaStreamSynchronize(st));
}

}  // namespace sapb

// One system of a batch stack: row-major band rows scaled by `scale`,
// entries outside the system's columns [0, n) zeroed.
static __global__ void k_stack_rows(double* __restrict__ A, int n, int K, double scale) {
  const long long W = 2LL * K + 1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * W;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / W;
    const long long c = r + (e - r * W) - K;
    A[e] = (c >= 0 && c < n) ? A[e] * scale : 0.0;
  }
}

// Per-segment sums of squares: out[s] = sum over rows [seg[s], seg[s+1]) of
// r^2, one CTA per segment, fixed-order reduction.
static __global__ void k_seg_sumsq(const double* __restrict__ r, const long long* __restrict__ seg,
                                   double* __restrict__ out) {
  __shared__ double red[256];
  const long long a = seg[blockIdx.x], b = seg[blockIdx.x + 1];
  double s = 0;
  for (long long i = a + threadIdx.x; i < b; i += blockDim.x) s += r[i] * r[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// ===========================================================================
// C ABI
using namespace sapb;

struct sap_solver { std::unique_ptr<Solver> s; };
struct sap_banded { Banded b; };
struct sap_csr { Csr c; };
struct sap_spmv { Spmv op; cudaStream_t st = nullptr; };

#define SAP_TRY(...)                                     \
  try {                                                  \
    __VA_ARGS__;                                         \
    return SAP_OK;                                       \
  } catch (const sapb::Error& e) {                       \
    g_last_error = e.what();                             \
    return e.code;                                       \
  } catch (const std::bad_alloc&) {                      \
    g_last_error = "host allocation failed";             \
    return SAP_ERR_OUT_OF_MEMORY;                        \
  } catch (const std::exception& e) {                    \
    g_last_error = e.what();                             \
    return SAP_ERR_CUDA;                                 \
  }

#define SAP_REQUIRE(cond, msg) \
  do { if (!(cond)) throw sapb::Error(SAP_ERR_INVALID_ARGUMENT, msg); } while (0)

extern "C" {

const char* sap_last_error(void) { return g_last_error.c_str(); }
int64_t sap_kernel_launch_count(void) { return g_launches.load(); }
int64_t sap_library_call_count(void) { return g_lib_calls.load(); }

int sap_profile_select(const char* name) {
  SAP_TRY({
    std::lock_guard<std::mutex> lk(g_prof.mu);
    for (auto& pr : g_prof.pairs) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    g_prof.pairs.clear();
    g_prof.name = name ? name : "";
  });
}

int sap_profile_read(double* total_ms, int64_t* launches) {
  SAP_TRY({
    std::lock_guard<std::mutex> lk(g_prof.mu);
    double tot = 0;
    for (auto& pr : g_prof.pairs) {
      SAPB_CUDA(cudaEventSynchronize(pr.second));
      float ms = 0;
      SAPB_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
      tot += ms;
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = (int64_t)g_prof.pairs.size();
  });
}

int sap_options_default(sap_options* o) {
  SAP_TRY({
    SAP_REQUIRE(o, "null options");
    std::memset(o, 0, sizeof(*o));
    o->solverType = SAP_BICGSTAB2;
    o->maxNumIterations = 100;
    o->relTol = 1e-6;
    o->absTol = 0;
    o->performReorder = 1;
    o->performDB = 1;
    o->applyScaling = 1;
    o->maxBandwidth = std::numeric_limits<int>::max();
    o->gpuCount = 1;
    o->dropOffFraction = 0;
    o->factMethod = SAP_LU_ONLY;
    o->precondType = SAP_PRECOND_SPIKE;
    o->variableBandwidth = 1;
    o->ilu_level = -1;
  });
}

int sap_banded_create(int n, int k, const double* data, int memspace, sap_banded** out) {
  SAP_TRY({
    SAP_REQUIRE(out && data && n > 0 && k >= 0 && k < n, "invalid banded matrix arguments");
    auto h = std::make_unique<sap_banded>();
    h->b.n = n; h->b.K = k;
    size_t cnt = (size_t)n * (2 * k + 1);
    h->b.A.alloc(cnt);
    SAPB_CUDA(cudaMemcpy(h->b.A.get(), data, cnt * sizeof(double),
                         memspace == SAP_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    *out = h.release();
  });
}

int sap_banded_generate(int n, int k, double d, int dist, uint64_t seed, sap_banded** out) {
  SAP_TRY({
    SAP_REQUIRE(out && n > 0 && k >= 0 && k < n && dist >= 0 && dist <= 2, "invalid generator arguments");
    std::vector<double> h((size_t)n * (2 * k + 1), 0.0);
    sapb::generate_band(n, k, d, dist, seed, h.data());
    auto m = std::make_unique<sap_banded>();
    m->b.n = n; m->b.K = k;
    m->b.A.alloc(h.size());
    SAPB_CUDA(cudaMemcpy(m->b.A.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    *out = m.release();
  });
}

int sap_generate_band_host(int n, int k, double d, int dist, uint64_t seed, double* out) {
  SAP_TRY({
    SAP_REQUIRE(out && n > 0 && k >= 0 && k < n && dist >= 0 && dist <= 2, "invalid generator arguments");
    std::memset(out, 0, sizeof(double) * (size_t)n * (2 * k + 1));
    sapb::generate_band(n, k, d, dist, seed, out);
  });
}

int sap_banded_copy_out(const sap_banded* A, double* dst, int memspace) {
  SAP_TRY({
    SAP_REQUIRE(A && dst, "null argument");
    SAPB_CUDA(cudaMemcpy(dst, A->b.A.get(), A->b.A.size() * sizeof(double),
                         memspace == SAP_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
  });
}

int sap_banded_info(const sap_banded* A, int* n, int* k) {
  SAP_TRY({
    SAP_REQUIRE(A, "null matrix");
    if (n) *n = A->b.n;
    if (k) *k = A->b.K;
  });
}

int sap_banded_destroy(sap_banded* A) { delete A; return SAP_OK; }

int sap_csr_create(int n, int nnz, const int* rp, const int* ci, const double* v, int memspace, sap_csr** out) {
  SAP_TRY({
    SAP_REQUIRE(out && rp && ci && v && n > 0 && nnz >= 0, "invalid CSR arguments");
    auto h = std::make_unique<sap_csr>();
    h->c.n = n; h->c.nnz = nnz;
    h->c.rp_h.resize(n + 1); h->c.ci_h.resize(nnz); h->c.v_h.resize(nnz);
    if (memspace == SAP_DEVICE) {
      SAPB_CUDA(cudaMemcpy(h->c.rp_h.data(), rp, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost));
      SAPB_CUDA(cudaMemcpy(h->c.ci_h.data(), ci, (size_t)nnz * sizeof(int), cudaMemcpyDeviceToHost));
      SAPB_CUDA(cudaMemcpy(h->c.v_h.data(), v, (size_t)nnz * sizeof(double), cudaMemcpyDeviceToHost));
    } else {  // host copies in parallel chunks (the first touch of the uninitialised vectors)
      _Pragma("omp parallel for schedule(static)")
      for (int c = 0; c < 64; c++) {
        const long long a = (long long)nnz * c / 64, e = (long long)nnz * (c + 1) / 64;
        const long long ra = (long long)(n + 1) * c / 64, re = (long long)(n + 1) * (c + 1) / 64;
        std::copy(rp + ra, rp + re, h->c.rp_h.begin() + ra);
        std::copy(ci + a, ci + e, h->c.ci_h.begin() + a);
        std::copy(v + a, v + e, h->c.v_h.begin() + a);
      }
    }
    SAP_REQUIRE(h->c.rp_h[0] == 0 && h->c.rp_h[n] == nnz, "row offsets inconsistent with nnz");
    int bad_rp = 0, bad_ci = 0;
    _Pragma("omp parallel for schedule(static) reduction(| : bad_rp)")
    for (int i = 0; i < n; i++) bad_rp |= h->c.rp_h[i] > h->c.rp_h[i + 1];
    SAP_REQUIRE(!bad_rp, "row offsets not monotone");
    _Pragma("omp parallel for schedule(static) reduction(| : bad_ci)")
    for (int p = 0; p < nnz; p++) bad_ci |= h->c.ci_h[p] < 0 || h->c.ci_h[p] >= n;
    SAP_REQUIRE(!bad_ci, "column index out of range");
    h->c.rp.upload(h->c.rp_h.data(), h->c.rp_h.size(), nullptr);
    h->c.ci.upload(h->c.ci_h.data(), h->c.ci_h.size(), nullptr);
    h->c.v.upload(h->c.v_h.data(), h->c.v_h.size(), nullptr);
    {
      const std::vector<int> blk = csr_row_blocks(n, h->c.rp_h.data());
      h->c.nblk = (int)blk.size() - 1;
      h->c.blk.upload(blk, nullptr);
    }
    SAPB_CUDA(cudaDeviceSynchronize());
    *out = h.release();
  });
}

int sap_csr_info(const sap_csr* A, int* n, int* nnz) {
  SAP_TRY({
    SAP_REQUIRE(A, "null matrix");
    if (n) *n = A->c.n;
    if (nnz) *nnz = A->c.nnz;
  });
}

int sap_csr_destroy(sap_csr* A) { delete A; return SAP_OK; }

int sap_spmv_banded_create(const sap_banded* A, sap_spmv** out) {
  SAP_TRY({
    SAP_REQUIRE(A && out, "null argument");
    auto h = std::make_unique<sap_spmv>();
    h->op.kind = 0; h->op.band = &A->b; h->op.n = A->b.n;
    *out = h.release();
  });
}

int sap_spmv_csr_create(const sap_csr* A, sap_spmv** out) {
  SAP_TRY({
    SAP_REQUIRE(A && out, "null argument");
    auto h = std::make_unique<sap_spmv>();
    h->op.kind = 1; h->op.csr = &A->c; h->op.n = A->c.n;
    *out = h.release();
  });
}

int sap_spmv_callback_create(int n, sap_spmv_fn fn, void* ctx, sap_spmv** out) {
  SAP_TRY({
    SAP_REQUIRE(fn && out && n > 0, "invalid callback operator");
    auto h = std::make_unique<sap_spmv>();
    h->op.kind = 2; h->op.fn = fn; h->op.ctx = ctx; h->op.n = n;
    *out = h.release();
  });
}

int sap_spmv_apply(sap_spmv* op, const double* x, double* y) {
  SAP_TRY({
    SAP_REQUIRE(op && x && y, "null argument");
    op->op.apply(x, y, nullptr);
    SAPB_CUDA(cudaStreamSynchronize(nullptr));
  });
}

int sap_spmv_destroy(sap_spmv* op) { delete op; return SAP_OK; }

int sap_blas_dots(int n, int nq, const double* const* x, const double* const* y, double* out, void* stream) {
  SAP_TRY({
    SAP_REQUIRE(n >= 0 && nq >= 1 && nq <= 4 && x && y && out, "invalid dot-product arguments");
    DotArgs a{};
    a.nq = nq;
    for (int q = 0; q < nq; q++) {
      SAP_REQUIRE(x[q] && y[q], "null vector");
      a.x[q] = x[q];
      a.y[q] = y[q];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = dot_grid_for(n);
    double* part = nullptr;
    unsigned int* ctr = nullptr;
    SAPB_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * 4 * (size_t)grid, st));
    SAPB_CUDA(cudaMallocAsync((void**)&ctr, sizeof(unsigned int), st));
    SAPB_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned int), st));
    k_dots<<<grid, kDotThreads, 0, st>>>(n, a, part, ctr, out);
    SAPB_LAUNCHED();
    SAPB_CUDA(cudaFreeAsync(part, st));
    SAPB_CUDA(cudaFreeAsync(ctr, st));
  });
}

int sap_tc_gemm_batched(int m, int n, int k, float alpha, const float* A, int lda, long long sA, const float* B,
                        int ldb, long long sB, float beta, float* C, int ldc, long long sC, int batch, void* stream) {
  SAP_TRY({
    SAP_REQUIRE(m >= 0 && n >= 0 && k >= 0 && batch >= 0 && lda >= std::max(1, m) && ldb >= std::max(1, k) &&
                    ldc >= std::max(1, m) && A && B && C,
                "invalid GEMM arguments");
    if (!umma::available()) throw Error(SAP_ERR_UNSUPPORTED, "the tensor-core GEMM needs an sm_100 device");
    static DBuf<int> err;  // error word of the kernel's bounded waits (one per process)
    cudaStream_t st = (cudaStream_t)stream;
    if (err.size() == 0) {
      err.alloc(1);
      err.zero(st);
    }
    umma::prepare();
    if (!umma::gemm(m, n, k, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, err.get(), st))
      throw Error(SAP_ERR_UNSUPPORTED,
                  "operand views break the TMA rules (16-byte aligned bases, leading dimensions and batch strides "
                  "multiples of 4 values)");
    int e = 0;
    SAPB_CUDA(cudaMemcpyAsync(&e, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    SAPB_CUDA(cudaStreamSynchronize(st));
    if (e) {
      err.zero(st);
      throw Error(SAP_ERR_DEVICE_TIMEOUT, "a tensor-core GEMM wait ran out of its iteration limit");
    }
  });
}

int sap_solver_create(int P, const sap_options* opts, int prec_dtype, sap_solver** out) {
  SAP_TRY({
    SAP_REQUIRE(out && opts && P >= 1, "invalid solver arguments");
    SAP_REQUIRE(prec_dtype == SAP_PREC_FLOAT || prec_dtype == SAP_PREC_DOUBLE || prec_dtype == SAP_PREC_TF32 ||
                    prec_dtype == SAP_PREC_TF32_F16,
                "invalid preconditioner type");
    SAP_REQUIRE(opts->refinementSweeps >= 0, "refinementSweeps must be >= 0");
    auto h = std::make_unique<sap_solver>();
    h->s = std::make_unique<Solver>(P, *opts, prec_dtype);
    *out = h.release();
  });
}

int sap_solver_destroy(sap_solver* s) { delete s; return SAP_OK; }

static void finish_setup_stats(Solver& S, double t_setup) {
  auto& st = S.stats;
  auto& pc = S.pc();
  st.timeSetup = t_setup;
  st.bandwidthReorder = pc.k_reorder;
  st.bandwidthDB = pc.k_db;
  st.bandwidth = pc.K;
  st.numPartitions = pc.P;
  st.actualDropOff = pc.drop_actual;
  st.time_toBanded = pc.t_toBanded;
  st.time_offDiags = pc.t_offDiags;
  st.time_bandLU = pc.t_bandLU;
  st.time_assembly = pc.t_assembly;
  st.time_fullLU = pc.t_fullLU;
  st.time_DB = pc.t_DB;
  st.time_reorder = pc.t_reorder;
  st.time_dropOff = pc.t_dropOff;
  st.time_cpu_assemble = pc.t_cpu_assemble;
  st.time_transfer = pc.t_transfer;
}

int sap_solver_setup_banded(sap_solver* h, const sap_banded* A) {
  SAP_TRY({
    SAP_REQUIRE(h && A, "null argument");
    Solver& S = *h->s;
    auto t0 = Clock::now();
    PrecBase& pc = S.pc();
    pc.reordered = false;
    pc.setup_rowmajor(A->b.A.get(), A->b.n, A->b.K);
    SAPB_CUDA(cudaStreamSynchronize(pc.st));
    S.n = pc.n;
    S.nnz = (long long)A->b.n * (2 * A->b.K + 1);
    S.setup_done = true;
    finish_setup_stats(S, ms_since(t0));
  });
}

int sap_solver_setup_csr(sap_solver* h, const sap_csr* A) {
  SAP_TRY({
    SAP_REQUIRE(h && A, "null argument");
    Solver& S = *h->s;
    auto t0 = Clock::now();
    PrecBase& pc = S.pc();
    if (!S.opts.performReorder) {
      // convertToBandedMatrix(CSR) (sap/precond.h:2240-2368)
      pc.reordered = false;
      int K = 0;
      for (int i = 0; i < A->c.n; i++)
        for (int p = A->c.rp_h[i]; p < A->c.rp_h[i + 1]; p++) K = std::max(K, std::abs(i - A->c.ci_h[p]));
      pc.setup_csr_direct(A->c, K);
    } else {
      pc.setup_sparse(A->c);
    }
    SAPB_CUDA(cudaStreamSynchronize(pc.st));
    S.n = pc.n;
    S.nnz = A->c.nnz;
    S.setup_done = true;
    finish_setup_stats(S, ms_since(t0));
  });
}

int sap_solver_update(sap_solver* h, const double* entries, int64_t nnz, int memspace, int* accepted) {
  SAP_TRY({
    SAP_REQUIRE(h && entries, "null argument");
    Solver& S = *h->s;
    if (!S.setup_done) throw Error(SAP_ILLEGAL_UPDATE, "Illegal call to update() before setup().");
    if (!S.opts.trackReordering)
      throw Error(SAP_ILLEGAL_UPDATE, "Illegal call to update() with reordering tracking disabled.");
    if (nnz != S.nnz) {
      if (accepted) *accepted = 0;
      return SAP_OK;
    }
    auto t0 = Clock::now();
    PrecBase& pc = S.pc();
    pc.update_values(entries, nnz, memspace == SAP_DEVICE);
    SAPB_CUDA(cudaStreamSynchronize(S.st));
    // Solver::update statistics (sap/solver.h:440-460)
    S.stats.timeUpdate = ms_since(t0);
    S.stats.time_reorder = 0;
    S.stats.time_DB = 0;
    S.stats.time_dropOff = 0;
    S.stats.time_cpu_assemble = pc.t_cpu_assemble;
    S.stats.time_transfer = pc.t_transfer;
    S.stats.time_toBanded = pc.t_toBanded;
    S.stats.time_offDiags = pc.t_offDiags;
    S.stats.time_bandLU = pc.t_bandLU;
    S.stats.time_assembly = pc.t_assembly;
    S.stats.time_fullLU = pc.t_fullLU;
    if (accepted) *accepted = 1;
  });
}

int sap_solver_solve(sap_solver* h, sap_spmv* spmv, const double* b, double* x, int memspace, int* converged) {
  SAP_TRY({
    SAP_REQUIRE(h && spmv && b && x, "null argument");
    Solver& S = *h->s;
    if (!S.setup_done) throw Error(SAP_ILLEGAL_SOLVE, "Illegal call to solve() before setup().");
    SAP_REQUIRE(spmv->op.n == S.n, "operator size differs from the preconditioner's");
    int L = 0;
    if (S.opts.solverType == SAP_BICGSTAB2) L = 2;
    else if (S.opts.solverType == SAP_BICGSTAB1) L = 1;
    else if (S.opts.solverType == SAP_BICGSTAB) L = -1;
    else if (S.opts.solverType == SAP_MINRES) L = -2;
    else if (S.opts.solverType != SAP_FGMRES)
      throw Error(SAP_ERR_UNSUPPORTED, "the CUSP solvers (BiCGStab_C, GMRES_C, CG_C, CR_C) are not provided");
    auto t0 = Clock::now();
    const size_t bytes = (size_t)S.n * sizeof(double);
    S.bvec.alloc(S.n);
    S.xvec.alloc(S.n);
    cudaMemcpyKind kin = memspace == SAP_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    SAPB_CUDA(cudaMemcpyAsync(S.bvec.get(), b, bytes, kin, S.st));
    SAPB_CUDA(cudaMemcpyAsync(S.xvec.get(), x, bytes, kin, S.st));
    S.mon.init(S.nrm2(S.bvec.get()));
    if (S.opts.refinementSweeps > 0) S.refine(spmv->op, S.xvec.get(), S.bvec.get(), L, S.opts.refinementSweeps);
    else S.krylov(spmv->op, S.xvec.get(), S.bvec.get(), L);
    cudaMemcpyKind kout = memspace == SAP_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    SAPB_CUDA(cudaMemcpyAsync(x, S.xvec.get(), bytes, kout, S.st));
    SAPB_CUDA(cudaStreamSynchronize(S.st));
    S.pc().check_device();
    S.stats.timeSolve = ms_since(t0);
    S.stats.rhsNorm = S.mon.rhsNorm;
    S.stats.residualNorm = S.mon.rNorm;
    S.stats.relResidualNorm = S.mon.rNorm / S.mon.rhsNorm;
    S.stats.numIterations = S.mon.it;
    if (converged) *converged = S.mon.code > 0 ? 1 : 0;
  });
}

int sap_precond_apply(sap_solver* h, const double* v, double* z) {
  SAP_TRY({
    SAP_REQUIRE(h && v && z, "null argument");
    Solver& S = *h->s;
    if (!S.setup_done) throw Error(SAP_ILLEGAL_SOLVE, "preconditioner used before setup().");
    S.pc().apply(v, z);
    SAPB_CUDA(cudaStreamSynchronize(S.st));
    S.pc().check_device();
  });
}

// Batched solve of independent banded systems (no reference counterpart).
// Systems with the same half-bandwidth are stacked into one block-diagonal
// banded system (entries of a system never reach another: its band rows
// have zeros outside its own columns), each system's rows scaled by
// 1/||b_i|| so that the stacked right-hand side has unit blocks; the stack
// is set up and solved once, to the absolute residual relTol, which bounds
// every block: ||r_i|| <= relTol ||b_i||.  The partition count of a stack is
// the sum of the systems' own counts.
int sap_batch_banded_solve(int m, const int* n, const int* k, const double* const* bands, const double* const* b,
                           double* const* x, int num_partitions, const sap_options* opts, int prec_dtype,
                           sap_batch_result* results, double* seconds) {
  SAP_TRY({
    SAP_REQUIRE(m > 0 && n && k && bands && b && x && opts && results, "null or empty batch");
    for (int i = 0; i < m; i++) SAP_REQUIRE(n[i] > 0 && k[i] >= 0 && k[i] < n[i] && bands[i] && b[i] && x[i], "bad system");
    auto t0 = Clock::now();
    std::vector<int> order(m);
    for (int i = 0; i < m; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return k[a] < k[c]; });
    size_t g0 = 0;
    while (g0 < order.size()) {
      size_t g1 = g0;
      const int K = k[order[g0]];
      while (g1 < order.size() && k[order[g1]] == K) g1++;
      // stack the group
      long long ntot = 0;
      int Ptot = 0;
      std::vector<long long> seg{0};
      std::vector<double> scale;
      for (size_t q = g0; q < g1; q++) {
        const int i = order[q];
        ntot += n[i];
        seg.push_back(ntot);
        double bn = 0;
        for (int r = 0; r < n[i]; r++) bn += b[i][r] * b[i][r];
        bn = std::sqrt(bn);
        scale.push_back(bn > 0 ? 1.0 / bn : 1.0);
        Ptot += std::max(1, std::min(num_partitions, n[i] / std::max(K + 1, 2 * K)));
      }
      SAP_REQUIRE(ntot < 2147483647LL, "stacked system too large");
      const size_t W = 2 * (size_t)K + 1;
      std::vector<double> bb((size_t)ntot), xx((size_t)ntot, 0.0);
      // the stack on the device: every system copied into its rows, then
      // scaled, with the entries outside its own columns dropped so that no
      // system reaches into its neighbours
      auto Ah = std::make_unique<sap_banded>();
      Ah->b.n = (int)ntot;
      Ah->b.K = K;
      Ah->b.A.alloc((size_t)ntot * W);
      for (size_t q = g0; q < g1; q++) {
        const int i = order[q];
        const long long off = seg[q - g0];
        SAPB_CUDA(cudaMemcpy(Ah->b.A.get() + (size_t)off * W, bands[i], sizeof(double) * (size_t)n[i] * W,
                             cudaMemcpyHostToDevice));
        k_stack_rows<<<grid_for((long long)n[i] * (long long)W, 256), 256>>>(Ah->b.A.get() + (size_t)off * W, n[i], K,
                                                                             scale[q - g0]);
        SAPB_LAUNCHED();
        const double sc = scale[q - g0];
        for (int r = 0; r < n[i]; r++) bb[off + r] = b[i][r] * sc;
      }
      SAPB_CUDA(cudaDeviceSynchronize());
      sap_options o = *opts;
      o.absTol = opts->relTol;
      o.relTol = 0;
      o.performReorder = 0;
      o.variableBandwidth = 0;
      o.applyScaling = 0;
      sap_banded* A = Ah.release();
      sap_spmv* op = nullptr;
      sap_solver* sv = nullptr;
      int rc = sap_spmv_banded_create(A, &op);
      if (rc == SAP_OK) rc = sap_solver_create(Ptot, &o, prec_dtype, &sv);
      if (rc == SAP_OK) rc = sap_solver_setup_banded(sv, A);
      int conv = 0;
      if (rc == SAP_OK) rc = sap_solver_solve(sv, op, bb.data(), xx.data(), SAP_HOST, &conv);
      if (rc == SAP_OK) {
        // per-system residual norms of the scaled stack = relative residuals
        Solver& S = *sv->s;
        DBuf<double> xd, rd, sq;
        DBuf<long long> segd;
        xd.upload(xx, S.st);
        rd.alloc((size_t)ntot);
        sq.alloc(g1 - g0);
        segd.upload(seg, S.st);
        op->op.apply(xd.get(), rd.get(), S.st);
        DBuf<double> bd;
        bd.upload(bb, S.st);
        k_axpby<<<grid_for(ntot, 256), 256, 0, S.st>>>((int)ntot, 1.0, bd.get(), -1.0, rd.get(), rd.get());
        SAPB_LAUNCHED();
        k_seg_sumsq<<<(int)(g1 - g0), 256, 0, S.st>>>(rd.get(), segd.get(), sq.get());
        SAPB_LAUNCHED();
        std::vector<double> sqh;
        sq.download(sqh, S.st);
        SAPB_CUDA(cudaStreamSynchronize(S.st));
        for (size_t q = g0; q < g1; q++) {
          const int i = order[q];
          results[i].rel_residual = std::sqrt(sqh[q - g0]);
          results[i].iterations = S.stats.numIterations;
          results[i].converged = results[i].rel_residual <= opts->relTol ? 1 : 0;
          std::memcpy(x[i], xx.data() + seg[q - g0], sizeof(double) * n[i]);
        }
      }
      if (sv) sap_solver_destroy(sv);
      if (op) sap_spmv_destroy(op);
      if (A) sap_banded_destroy(A);
      if (rc != SAP_OK) return rc;
      g0 = g1;
    }
    if (seconds) *seconds = ms_since(t0) / 1e3;
  });
}

int sap_solver_get_stats(const sap_solver* h, sap_stats* out) {
  SAP_TRY({
    SAP_REQUIRE(h && out, "null argument");
    *out = h->s->stats;
  });
}

int sap_solver_get_monitor(const sap_solver* h, int* code, const char** message) {
  SAP_TRY({
    SAP_REQUIRE(h, "null argument");
    if (code) *code = h->s->mon.code;
    if (message) *message = h->s->mon.msg.c_str();
  });
}

int sap_solver_info(const sap_solver* h, int* n, int* k, int* P) {
  SAP_TRY({
    SAP_REQUIRE(h, "null argument");
    if (n) *n = h->s->pcp->n;
    if (k) *k = h->s->pcp->K;
    if (P) *P = h->s->pcp->P;
  });
}

int sap_solver_block_layout(const sap_solver* h, int* block_size, int* blocks_per_partition, int* value_bytes) {
  SAP_TRY({
    SAP_REQUIRE(h, "null argument");
    const PrecBase& pc = *h->s->pcp;
    int bs = 0, nb = 0;
    pc.block_layout(bs, nb);
    if (block_size) *block_size = bs;
    if (blocks_per_partition) *blocks_per_partition = nb;
    if (value_bytes)
      *value_bytes = h->s->prec_dtype == SAP_PREC_DOUBLE ? 8 : (h->s->prec_dtype == SAP_PREC_TF32_F16 && bs > 0 ? 2 : 4);
  });
}

int sap_solver_get_reorder(const sap_solver* h, int which, int* out, int64_t* count) {
  SAP_TRY({
    SAP_REQUIRE(h && count, "null argument");
    const PrecBase& pc = *h->s->pcp;
    const std::vector<int>* v = nullptr;
    switch (which) {
      case 0: v = &pc.db_row_perm_h; break;
      case 1: v = &pc.final_pos_h; break;
      case 2: v = &pc.final_order_h; break;
      case 3: v = &pc.first_rows_h; break;
      case 4: v = &pc.part_k_h; break;
      default: throw Error(SAP_ERR_INVALID_ARGUMENT, "unknown reorder array");
    }
    *count = (int64_t)v->size();
    if (out) std::copy(v->begin(), v->end(), out);
  });
}

void* sap_solver_stream(const sap_solver* h) { return h ? (void*)h->s->st : nullptr; }

}  // extern "C"
