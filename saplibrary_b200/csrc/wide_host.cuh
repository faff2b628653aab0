// Host side of the wide-band path (see wide_band.cuh): block storage,
// recursive block LU with triangular inverses, spike tips and the reduced
// system as batched matrix products, and the block-row sweeps.
#pragma once

#include <cublas_v2.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "common.cuh"
#include "umma_gemm.cuh"
#include "wide_band.cuh"

namespace sapb {

inline void cublas_check(cublasStatus_t s, const char* what) {
  if (s != CUBLAS_STATUS_SUCCESS) throw Error(SAP_ERR_CUDA, std::string(what) + ": cuBLAS status " + std::to_string((int)s));
}

// Strided-batched column-major GEMM, C = alpha A B + beta C (plain library GEMM).
template <typename T>
struct Gemm;
template <>
struct Gemm<double> {
  static void run(cublasHandle_t h, int m, int n, int k, double alpha, const double* A, int lda, long long sA,
                  const double* B, int ldb, long long sB, double beta, double* C, int ldc, long long sC, int batch) {
    if (m <= 0 || n <= 0 || batch <= 0) return;
    cublas_check(cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &alpha, A, lda, sA, B, ldb, sB, &beta,
                                           C, ldc, sC, batch),
                 "cublasDgemmStridedBatched");
    count_lib_call();
  }
};
template <>
struct Gemm<float> {
  static void run(cublasHandle_t h, int m, int n, int k, float alpha, const float* A, int lda, long long sA,
                  const float* B, int ldb, long long sB, float beta, float* C, int ldc, long long sC, int batch) {
    if (m <= 0 || n <= 0 || batch <= 0) return;
    cublas_check(cublasSgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &alpha, A, lda, sA, B, ldb, sB, &beta,
                                           C, ldc, sC, batch),
                 "cublasSgemmStridedBatched");
    count_lib_call();
  }
};

// A batch of equally strided column-major matrices.
template <typename T>
struct Mat {
  T* p;
  int ld;
  long long s;  // batch stride
  Mat at(int r, int c) const { return Mat{p + (long long)c * ld + r, ld, s}; }
};

template <typename T>
class BlockLU {
 public:
  cublasHandle_t h = nullptr;
  cudaStream_t st = nullptr;
  int batch = 0;
  bool boost = true;
  int* flag = nullptr;
  Mat<T> W;  // workspace, >= n x n per batch element (the inverse-block temporaries of rec)

  // tc: TF32 products on this library's tensor-core kernel (umma::gemm);
  // otherwise, and for a view that does not meet the TMA rules, cuBLAS
  bool tc = false;
  int* gerr = nullptr;  // error word of the tensor-core kernel's bounded waits
  void gemm(int m, int n, int k, T alpha, Mat<T> A, Mat<T> B, T beta, Mat<T> C) {
    if constexpr (sizeof(T) == 4) {
      if (tc && umma::gemm(m, n, k, alpha, A.p, A.ld, A.s, B.p, B.ld, B.s, beta, C.p, C.ld, C.s, batch, gerr, st))
        return;
    }
    Gemm<T>::run(h, m, n, k, alpha, A.p, A.ld, A.s, B.p, B.ld, B.s, beta, C.p, C.ld, C.s, batch);
  }
  void copy(Mat<T> src, Mat<T> dst, int m, int n, T scale = T(1)) {
    if (m <= 0 || n <= 0) return;
    dim3 g((m + 255) / 256, std::min(n, 1024), batch);
    k_sub_copy<T><<<g, 256, 0, st>>>(src.p, src.ld, src.s, dst.p, dst.ld, dst.s, m, n, scale);
    SAPB_LAUNCHED();
  }

  void fill(Mat<T> dst, int m, int n, T value) {
    if (m <= 0 || n <= 0) return;
    dim3 g((m + 255) / 256, std::min(n, 1024), batch);
    k_sub_fill<T><<<g, 256, 0, st>>>(dst.p, dst.ld, dst.s, m, n, value);
    SAPB_LAUNCHED();
  }

  // Products with triangular operands, recursing on halves and skipping the
  // structurally zero quarter (the skipped terms are exact zeros, so the
  // results equal the full products up to summation order).  Below `cut`
  // a full GEMM.  C never aliases A or B.  L: lower, U: upper, F: full.
  int cut = 384;  // WideBand sets it: recursion pays off for compute-bound FP64 / FP32, not for TF32
  static int half(int n) { return std::max(32, ((n / 2 + 31) / 32) * 32); }
  // C (n x m) = alpha L B + beta C
  void prod_LF(int n, int m, T alpha, Mat<T> L, Mat<T> B, T beta, Mat<T> C) {
    if (n <= cut) return gemm(n, m, n, alpha, L, B, beta, C);
    const int n1 = half(n), n2 = n - n1;
    prod_LF(n1, m, alpha, L, B, beta, C);
    gemm(n2, m, n1, alpha, L.at(n1, 0), B, beta, C.at(n1, 0));
    prod_LF(n2, m, alpha, L.at(n1, n1), B.at(n1, 0), T(1), C.at(n1, 0));
  }
  // C (n x m) = alpha U B + beta C
  void prod_UF(int n, int m, T alpha, Mat<T> U, Mat<T> B, T beta, Mat<T> C) {
    if (n <= cut) return gemm(n, m, n, alpha, U, B, beta, C);
    const int n1 = half(n), n2 = n - n1;
    prod_UF(n1, m, alpha, U, B, beta, C);
    gemm(n1, m, n2, alpha, U.at(0, n1), B.at(n1, 0), T(1), C);
    prod_UF(n2, m, alpha, U.at(n1, n1), B.at(n1, 0), beta, C.at(n1, 0));
  }
  // C (m x n) = alpha A U + beta C
  void prod_FU(int m, int n, T alpha, Mat<T> A, Mat<T> U, T beta, Mat<T> C) {
    if (n <= cut) return gemm(m, n, n, alpha, A, U, beta, C);
    const int n1 = half(n), n2 = n - n1;
    prod_FU(m, n1, alpha, A, U, beta, C);
    gemm(m, n2, n1, alpha, A, U.at(0, n1), beta, C.at(0, n1));
    prod_FU(m, n2, alpha, A.at(0, n1), U.at(n1, n1), T(1), C.at(0, n1));
  }
  // C (m x n) = alpha A L + beta C
  void prod_FL(int m, int n, T alpha, Mat<T> A, Mat<T> L, T beta, Mat<T> C) {
    if (n <= cut) return gemm(m, n, n, alpha, A, L, beta, C);
    const int n1 = half(n), n2 = n - n1;
    prod_FL(m, n1, alpha, A, L, beta, C);
    gemm(m, n1, n2, alpha, A.at(0, n1), L.at(n1, 0), T(1), C);
    prod_FL(m, n2, alpha, A.at(0, n1), L.at(n1, n1), beta, C.at(0, n1));
  }
  // C (lower, n x n) = alpha A B, A and B lower; C's upper part set to zero
  void prod_LL(int n, T alpha, Mat<T> A, Mat<T> B, Mat<T> C) {
    if (n <= cut) return gemm(n, n, n, alpha, A, B, T(0), C);
    const int n1 = half(n), n2 = n - n1;
    prod_LL(n1, alpha, A, B, C);
    fill(C.at(0, n1), n1, n2, T(0));
    prod_FL(n2, n1, alpha, A.at(n1, 0), B, T(0), C.at(n1, 0));
    prod_LF(n2, n1, alpha, A.at(n1, n1), B.at(n1, 0), T(1), C.at(n1, 0));
    prod_LL(n2, alpha, A.at(n1, n1), B.at(n1, n1), C.at(n1, n1));
  }
  // C (upper, n x n) = alpha A B, A and B upper; C's lower part set to zero
  void prod_UU(int n, T alpha, Mat<T> A, Mat<T> B, Mat<T> C) {
    if (n <= cut) return gemm(n, n, n, alpha, A, B, T(0), C);
    const int n1 = half(n), n2 = n - n1;
    prod_UU(n1, alpha, A, B, C);
    prod_UF(n1, n2, alpha, A, B.at(0, n1), T(0), C.at(0, n1));
    prod_FU(n1, n2, alpha, A.at(0, n1), B.at(n1, n1), T(1), C.at(0, n1));
    fill(C.at(n1, 0), n2, n1, T(0));
    prod_UU(n2, alpha, A.at(n1, n1), B.at(n1, n1), C.at(n1, n1));
  }
  // C (n x n) += alpha A B, A upper, B lower
  void prod_UL_acc(int n, T alpha, Mat<T> A, Mat<T> B, Mat<T> C) {
    if (n <= cut) return gemm(n, n, n, alpha, A, B, T(1), C);
    const int n1 = half(n), n2 = n - n1;
    prod_UL_acc(n1, alpha, A, B, C);
    gemm(n1, n1, n2, alpha, A.at(0, n1), B.at(n1, 0), T(1), C);
    prod_FL(n1, n2, alpha, A.at(0, n1), B.at(n1, n1), T(1), C.at(0, n1));
    prod_UF(n2, n1, alpha, A.at(n1, n1), B.at(n1, 0), T(1), C.at(n1, 0));
    prod_UL_acc(n2, alpha, A.at(n1, n1), B.at(n1, n1), C.at(n1, n1));
  }

  // Second lane: the two independent products of every recursion step (the
  // U12 / L21 panels, then the two off-diagonal inverse blocks) run on it
  // concurrently with the first; it has its own cuBLAS handle and workspace.
  cublasHandle_t h2 = nullptr;
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  void fork() {
    if (!st2) return;
    SAPB_CUDA(cudaEventRecord(ev_a, st));
    SAPB_CUDA(cudaStreamWaitEvent(st2, ev_a, 0));
  }
  void join() {
    if (!st2) return;
    SAPB_CUDA(cudaEventRecord(ev_b, st2));
    SAPB_CUDA(cudaStreamWaitEvent(st, ev_b, 0));
  }
  template <class F>
  void lane2(F&& f) {
    if (!st2) return f();
    struct Swap {
      BlockLU* b;
      explicit Swap(BlockLU* b_) : b(b_) { flip(); }
      ~Swap() { flip(); }
      void flip() {
        std::swap(b->h, b->h2);
        std::swap(b->st, b->st2);
      }
    } guard(this);
    f();
  }

  // Recursion workspace: every step keeps its U12 and L21 panels until its
  // inverse blocks are formed; rw holds them level by level (rec_ws(n)
  // values per batch element for an n x n factorization, batch stride rws).
  T* rw = nullptr;
  long long rws = 0;
  static int split(int n) {
    int n1 = ((n / 2 + kLeaf - 1) / kLeaf) * kLeaf;
    if (n1 >= n) n1 = n - kLeaf;
    return n1;
  }
  int leaf = leaf_size<T>();  // largest leaf of the recursion
  // leading dimension of an n-row workspace panel: a multiple of 4 values,
  // so that every panel view meets the TMA rules of the tensor-core GEMM
  static int pad4(int n) { return (n + 3) / 4 * 4; }
  static long long rec_ws(int n, int leaf) {
    if (n <= leaf) return 0;
    const int n1 = split(n), n2 = n - n1;
    return std::max(rec_ws(n1, leaf), (long long)n1 * n2 + (long long)pad4(n2) * n1 + rec_ws(n2, leaf));
  }
  template <int NL>
  void leaf_launch(Mat<T> M, Mat<T> Li, Mat<T> Ui, int n) {
    using LS = LeafShape<T, NL>;
    static bool smem_set = false;  // first call runs outside any graph capture
    if (!smem_set) {
      SAPB_CUDA(cudaFuncSetAttribute(k_leaf_lu<T, NL, LS::RY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)LS::smem));
      smem_set = true;
    }
    SAPB_PROF("wb_leaf", st);
    k_leaf_lu<T, NL, LS::RY><<<batch, LS::RY * 32, LS::smem, st>>>(M.p, M.ld, M.s, Li.p, Ui.p, Li.ld, Li.s, n,
                                                                    boost ? 1 : 0, flag);
    SAPB_LAUNCHED();
  }

  // Li = L^-1, Ui = U^-1 of M = L U (n x n at M; Li, Ui pre-zeroed).  M's
  // trailing blocks are overwritten by the Schur complements.  wo: this
  // level's offset into rw.
  void rec(Mat<T> M, Mat<T> Li, Mat<T> Ui, int n, long long wo = 0) {
    if (n <= leaf) {
      if (Li.s != Ui.s || Li.ld != Ui.ld) throw Error(SAP_ERR_INVALID_ARGUMENT, "leaf inverse layouts differ");
      if (leaf <= 32) leaf_launch<32>(M, Li, Ui, n);
      else if (leaf <= 64 || sizeof(T) != 4) leaf_launch<64>(M, Li, Ui, n);
      else leaf_launch<(sizeof(T) == 4 ? 128 : 64)>(M, Li, Ui, n);
      return;
    }
    const int n1 = split(n), n2 = n - n1;
    rec(M, Li, Ui, n1, wo);
    // U12 = L11^-1 A12, L21 = A21 U11^-1 (independent); A22 -= L21 U12
    const Mat<T> U12{rw + wo, n1, rws}, L21{rw + wo + (long long)n1 * n2, pad4(n2), rws};
    fork();
    prod_LF(n1, n2, T(1), Li, M.at(0, n1), T(0), U12);
    lane2([&] { prod_FU(n2, n1, T(1), M.at(n1, 0), Ui, T(0), L21); });
    join();
    gemm(n2, n2, n1, T(-1), L21, U12, T(1), M.at(n1, n1));
    rec(M.at(n1, n1), Li.at(n1, n1), Ui.at(n1, n1), n2, wo + (long long)n1 * n2 + (long long)pad4(n2) * n1);
    // (L^-1)21 = -L22^-1 L21 L11^-1, (U^-1)12 = -U11^-1 U12 U22^-1 (independent)
    const Mat<T> Tl{W.p, pad4(n2), W.s}, Tu{W.p + (long long)pad4(n2) * n1, n1, W.s};
    fork();
    prod_FL(n2, n1, T(1), L21, Li, T(0), Tl);
    prod_LF(n2, n1, T(-1), Li.at(n1, n1), Tl, T(0), Li.at(n1, 0));
    lane2([&] {
      prod_FU(n1, n2, T(1), U12, Ui.at(n1, n1), T(0), Tu);
      prod_UF(n1, n2, T(-1), Ui, Tu, T(0), Ui.at(0, n1));
    });
    join();
  }
};


inline int grid1d(long long work, int threads = 256, int cap = 148 * 32) {
  return (int)std::max<long long>(1, std::min<long long>((work + threads - 1) / threads, cap));
}

// Wide-band preconditioner state: the partitions' block LU (as inverses of
// the diagonal factors plus the off-diagonal factor blocks), the spike tips
// and the factored reduced system, and the apply.
template <typename T>
class WideBand {
 public:
  cublasHandle_t h = nullptr;
  cudaStream_t st = nullptr;
  int n = 0, P = 0, bs = 0, nb = 0, K = 0;  // K: width of the coupling blocks
  int ldK = 0;                               // leading dimension of the K x K blocks (16-byte multiple)
  long long sK = 0;                          // their batch stride, ldK * K
  bool spike = false;
  long long plen = 0, BB = 0;
  std::vector<int> pstart_h, psize_h;
  DBuf<int> pstart_d, psize_d, rowpart_d;
  DBuf<T> Linv, Uinv, Uoff, Loff;  // [P][nb] / [P][nb-1] blocks of bs x bs
  DBuf<T> Vc, Wc, Bc, Cc, SLi, SUi;  // [P-1] column-major K x K
  DBuf<long long> ipos, irow;        // interface unknowns: block-vector position / band row
  DBuf<T> Fb, xv, yv, tv, xbt, fbt, t1, t2;
  DBuf<int> flag;
  // setup workspaces, kept (with everything above) across setups of the
  // same layout so that a repeated setup does not free and re-allocate
  DBuf<T> Dw, Ww, X, Wt, S, Ws;
  DBuf<T> Rw, Rs;  // recursion workspaces of the partition factors / the reduced system
  DBuf<int> nz_d, spk_cols[2], spk_pos[2], sflag;  // spike-tip setup scratch

  // device bytes this object holds
  size_t bytes_held() const {
    size_t b = 0;
    for (const DBuf<T>* d : {&Linv, &Uinv, &Uoff, &Loff, &Vc, &Wc, &Bc, &Cc, &SLi, &SUi, &Fb, &xv, &yv, &tv, &xbt, &fbt,
                             &t1, &t2, &Dw, &Ww, &X, &Wt, &S, &Ws, &Rw, &Rs, &gws[0], &gws[1], &gws[2], &gws[3], &pws, &csL, &csU,
                             &csLo, &csUo})
      b += d->size() * sizeof(T);
    for (const DBuf<__half>* d : {&Lh, &Uh, &Loh, &Uoh}) b += d->size() * sizeof(__half);
    return b;
  }

  WideBand() = default;
  WideBand(const WideBand&) = delete;
  WideBand& operator=(const WideBand&) = delete;
  ~WideBand() {
    if (fgraph) cudaGraphExecDestroy(fgraph);
    if (st2) cudaStreamSynchronize(st2);
    for (cudaStream_t x : st_more)
      if (x) cudaStreamSynchronize(x);
    if (h) cublasDestroy(h);
    if (h2) cublasDestroy(h2);
    if (st2) cudaStreamDestroy(st2);
    for (cudaStream_t x : st_more)
      if (x) cudaStreamDestroy(x);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_half) cudaEventDestroy(ev_half);
    for (cudaEvent_t e : ev_lane)
      if (e) cudaEventDestroy(e);
  }

  // The factorization's launch sequence (about a thousand small GEMMs,
  // copies and leaf LUs per block row) as a CUDA graph: the first setup of a
  // layout runs it directly, the second captures it, later ones replay it
  // (every buffer it touches is kept across setups of the layout).
  cudaGraphExec_t fgraph = nullptr;
  long long fgraph_key = -1;
  int fgraph_cut = 0, fgraph_leaf = 0;
  // SAPB_FACTOR_GRAPH=0 runs the factorization's launches directly every time
  static bool graph_enabled() {
    const char* e = std::getenv("SAPB_FACTOR_GRAPH");
    return !(e && std::atoi(e) == 0);
  }
  int fgraph_runs = 0;
  bool fgraph_failed = false;
  int64_t fgraph_launches = 0, fgraph_lib_calls = 0;
  DBuf<unsigned char> cublas_ws, cublas_ws2;  // fixed cuBLAS workspaces (no allocation inside a capture)
  cublasHandle_t h2 = nullptr;                  // bound to st2 (second lane of the factorization)

  // Block size bs >= the largest half-bandwidth, a multiple of the leaf size.
  // Larger blocks mean fewer block rows, hence fewer dependent launches per
  // partition, for more factor flops and sweep bytes; with the tensor-core
  // TF32 products the flops are cheap and bs is at least 448 (2M-row K = 200
  // workload, TF32 + FGMRES: 0.154 s at bs 448 against 0.221 / 0.179 / 0.182 s
  // at 224 / 672 / 896; FP32 and FP64 are fastest at the smallest bs).
  // SAPB_BLOCK_SIZE raises it further.
  static int block_size(int kmax, bool tf32_products = false) {
    int bs = std::max(kLeaf, ((kmax + kLeaf - 1) / kLeaf) * kLeaf);
    if (tf32_products) bs = std::max(bs, 448);
    const char* e = std::getenv("SAPB_BLOCK_SIZE");
    if (e && std::atoi(e) > bs) bs = ((std::atoi(e) + kLeaf - 1) / kLeaf) * kLeaf;
    return bs;
  }

  // Device bytes of the factors, their FP16 copies (h16) and the
  // factorization workspaces for n rows in P partitions (for the memory check).
  static double factor_bytes(int n, int P, int kmax, bool h16 = false, bool tf32_products = false) {
    const double b = block_size(kmax, tf32_products);
    const double nbp = std::ceil((double)(n / P + 1) / b);
    return ((4.0 * nbp + 3.0) * sizeof(T) + (h16 ? 4.0 * nbp * 2.0 : 0.0)) * P * b * b;
  }

  // tf32: FP32 block products on the tensor cores (TF32 inputs, FP32
  // accumulation) for the partition factors, spikes and reduced systems.
  bool tf32 = false;
  // The TF32 products run on this library's tcgen05 kernel (umma_gemm.cuh)
  // on sm_100; SAPB_TC_GEMM=0 hands them to cuBLAS's TF32 mode instead.
  static bool tc_gemm_enabled() {
    const char* e = std::getenv("SAPB_TC_GEMM");
    return !(e && std::atoi(e) == 0) && umma::available();
  }
  bool tc_on() const { return tf32 && tc_gemm_enabled(); }
  DBuf<int> gemm_err;
  // after a synchronisation: a bounded wait of the tensor-core kernel that
  // ran out is reported (and the word cleared)
  void check_gemm() {
    if (gemm_err.size() == 0) return;
    int e = 0;
    SAPB_CUDA(cudaMemcpyAsync(&e, gemm_err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    SAPB_CUDA(cudaStreamSynchronize(st));
    if (e) {
      gemm_err.zero(st);
      SAPB_CUDA(cudaStreamSynchronize(st));
      throw Error(SAP_ERR_DEVICE_TIMEOUT, "a tensor-core GEMM wait ran out of its iteration limit");
    }
  }
  // h16: the block sweeps of the apply read FP16 copies of the factor
  // blocks with a power-of-two scale per column (half the bytes of FP32);
  // the setup keeps computing in FP32 / TF32.  FP32 storage only.
  bool h16 = false;
  DBuf<__half> Lh, Uh, Loh, Uoh;   // copies of Linv, Uinv, Loff, Uoff
  DBuf<T> csL, csU, csLo, csUo;    // their column scales ([block][bs])
  void make_half() {
    if (!h16) return;
    const long long nd = (long long)P * nb, no = (long long)P * (nb - 1);
    Lh.alloc((size_t)(nd * BB));
    Uh.alloc((size_t)(nd * BB));
    csL.alloc((size_t)(nd * bs));
    csU.alloc((size_t)(nd * bs));
    if (nb > 1) {
      Loh.alloc((size_t)(no * BB));
      Uoh.alloc((size_t)(no * BB));
      csLo.alloc((size_t)(no * bs));
      csUo.alloc((size_t)(no * bs));
    }
    // on the second stream, beside the spike products that follow on st
    // (both only read the factors); the apply and the next setup wait for it
    SAPB_CUDA(cudaEventRecord(ev_fork, st));
    SAPB_CUDA(cudaStreamWaitEvent(st2, ev_fork, 0));
    constexpr int R = tgemv_rows<T, 8>();  // rows per tile of the FP16 sweep kernel
    auto conv = [&](const T* A, __half* H, T* cs, long long nblk, int tri) {
      if (nblk <= 0) return;
      k_blocks_to_half<T, R><<<dim3((bs + 7) / 8, (unsigned)nblk), 256, 0, st2>>>(A, H, cs, bs, BB, tri);
      SAPB_LAUNCHED();
    };
    conv(Linv.get(), Lh.get(), csL.get(), nd, 1);
    conv(Uinv.get(), Uh.get(), csU.get(), nd, 2);
    if (nb > 1) {
      conv(Loff.get(), Loh.get(), csLo.get(), no, 2);
      conv(Uoff.get(), Uoh.get(), csUo.get(), no, 1);
    }
    SAPB_CUDA(cudaEventRecord(ev_half, st2));
    half_pending = true;
  }
  cudaEvent_t ev_half = nullptr;
  bool half_pending = false;
  // st waits for the FP16 conversion (before an apply reads the copies or a
  // setup overwrites the factors)
  void wait_half() {
    if (!half_pending) return;
    SAPB_CUDA(cudaStreamWaitEvent(st, ev_half, 0));
    half_pending = false;
  }
  // recursion cut-off of the spike slab products: structure-aware for the
  // compute-bound FP64 / FP32 products (FP64 spikes 0.99 -> 0.62 s on the
  // 1M-row workload), plain GEMMs for TF32; SAPB_SPIKE_CUT overrides
  int spike_cut() const {
    const char* e = std::getenv("SAPB_SPIKE_CUT");
    if (e && std::atoi(e) > 0) return std::atoi(e);
    return tf32 ? (1 << 30) : 384;
  }
  // The TF32 form builds and factors the reduced systems with TF32 products
  // too (1M-row workload: 41 -> 21 ms, the same 23 FGMRES iterations);
  // SAPB_REDUCED_TF32=0 keeps them in full FP32
  static bool reduced_tf32() {
    const char* e = std::getenv("SAPB_REDUCED_TF32");
    return !(e && std::atoi(e) == 0);
  }
  // the same cut-off for the products of the partition factorization: one
  // structure-aware level for TF32 (1M-row workload: block LU 187 -> 171 ms),
  // down to 384 for the compute-bound FP64 / FP32 products;
  // SAPB_FACTOR_CUT overrides
  int factor_cut() const {
    const char* e = std::getenv("SAPB_FACTOR_CUT");
    if (e && std::atoi(e) > 0) return std::atoi(e);
    return tf32 ? 2048 : 384;
  }
  void math_mode(bool fast) {
    for (cublasHandle_t x : {h, h2})
      cublas_check(cublasSetMathMode(x, fast ? CUBLAS_TF32_TENSOR_OP_MATH : CUBLAS_PEDANTIC_MATH), "cublasSetMathMode");
  }
  // the second lane of a recursive factorization, and the product engine
  void lanes(BlockLU<T>& lu) {
    lu.h2 = h2;
    lu.st2 = st2;
    lu.ev_a = ev_fork;
    lu.ev_b = ev_join;
    lu.tc = tc_on();
    lu.gerr = gemm_err.get();
  }

  void init(cudaStream_t s, int n_, int bs_, const std::vector<int>& pstart, const std::vector<int>& psize,
            bool tf32_ = false, bool h16_ = false) {
    st = s;
    tf32 = tf32_ && sizeof(T) == 4;
    h16 = h16_ && sizeof(T) == 4;
    n = n_;
    P = (int)pstart.size();
    bs = bs_;
    pstart_h = pstart;
    psize_h = psize;
    if (!h) cublas_check(cublasCreate(&h), "cublasCreate");
    if (!st2) {
      SAPB_CUDA(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
      SAPB_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
      SAPB_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
      for (cudaStream_t& x : st_more) SAPB_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
      for (cudaEvent_t& e : ev_lane) SAPB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      SAPB_CUDA(cudaEventCreateWithFlags(&ev_half, cudaEventDisableTiming));
    }
    wait_half();
    cublas_check(cublasSetStream(h, st), "cublasSetStream");
    if (cublas_ws.size() == 0) cublas_ws.alloc((size_t)64 << 20);
    cublas_check(cublasSetWorkspace(h, cublas_ws.get(), cublas_ws.size()), "cublasSetWorkspace");
    if (!h2) {
      cublas_check(cublasCreate(&h2), "cublasCreate");
      cublas_check(cublasSetStream(h2, st2), "cublasSetStream");
      cublas_ws2.alloc((size_t)32 << 20);
      cublas_check(cublasSetWorkspace(h2, cublas_ws2.get(), cublas_ws2.size()), "cublasSetWorkspace");
    }
    spike = false;
    math_mode(tf32);
    if (gemm_err.size() == 0) {
      gemm_err.alloc(1);
      gemm_err.zero(st);
    }
    if (tc_on()) umma::prepare();  // kernel attributes, before any capture
    int maxsz = 0;
    for (int v : psize) maxsz = std::max(maxsz, v);
    nb = std::max(1, (maxsz + bs - 1) / bs);
    plen = (long long)nb * bs;
    BB = (long long)bs * bs;
    pstart_d.upload(pstart, st);
    psize_d.upload(psize, st);
    std::vector<int> rowpart(n, 0);
    for (int p = 0; p < P; p++)
      for (int r = pstart[p]; r < pstart[p] + psize[p]; r++) rowpart[r] = p;
    rowpart_d.upload(rowpart, st);
    Linv.alloc((size_t)P * nb * BB);
    Uinv.alloc((size_t)P * nb * BB);
    Linv.zero(st);
    if (nb > 1) {
      Uoff.alloc((size_t)P * (nb - 1) * BB);
      Loff.alloc((size_t)P * (nb - 1) * BB);
      Uoff.zero(st);
      Loff.zero(st);
    }
    Fb.alloc(n);
    xv.alloc((size_t)P * plen);
    yv.alloc((size_t)P * plen);
    tv.alloc((size_t)P * plen);
  }

  Mat<T> blk(DBuf<T>& a, int per_part, int i) { return Mat<T>{a.get() + (long long)i * BB, bs, (long long)per_part * BB}; }

  // D_i land in the Linv slots, E_i in Uoff, F_i in Loff; padding rows get
  // an identity diagonal.
  void pad() {
    k_wb_pad<T><<<dim3(grid1d(plen, 256, 64), P), 256, 0, st>>>(Linv.get(), psize_d.get(), bs, nb);
    SAPB_LAUNCHED();
  }
  void load_band(const T* B, const std::vector<long long>& boff, const std::vector<int>& kp) {
    DBuf<long long> bo;
    DBuf<int> kd;
    bo.upload(boff, st);
    kd.upload(kp, st);
    int kmax = 0;
    for (int v : kp) kmax = std::max(kmax, v);
    k_wb_from_band<T><<<dim3(grid1d((long long)(n / P + 1) * (2 * kmax + 1), 256, 2048), P), 256, 0, st>>>(
        B, bo.get(), kd.get(), psize_d.get(), bs, nb, Linv.get(), Uoff.get(), Loff.get());
    SAPB_LAUNCHED();
    pad();
    SAPB_CUDA(cudaStreamSynchronize(st));
  }
  void load_coo(const int* rows, const int* cols, const T* vals, long long nz) {
    k_wb_scatter<T><<<grid1d(nz), 256, 0, st>>>(rows, cols, vals, nz, rowpart_d.get(), pstart_d.get(), psize_d.get(),
                                                 bs, nb, Linv.get(), Uoff.get(), Loff.get());
    SAPB_LAUNCHED();
    pad();
    SAPB_CUDA(cudaStreamSynchronize(st));
  }

  // Block-row LU of every partition, batched over the partitions:
  //   D_i <- D_i - L_{i,i-1} U_{i-1,i};  D_i = L_ii U_ii (recursive, with inverses);
  //   U_{i,i+1} = L_ii^-1 E_i;  L_{i+1,i} = F_i U_ii^-1.
  void factor(bool boost) {
    Dw.alloc((size_t)P * BB);
    Ww.alloc((size_t)P * BB);
    Rw.alloc((size_t)P * std::max(1LL, BlockLU<T>::rec_ws(bs, leaf_size<T>())));
    flag.alloc(1);
    const long long key = (((long long)P * 65537 + bs) * 65537 + nb) * 4 + (boost ? 2 : 0) + (tf32 ? 1 : 0);
    if (key != fgraph_key || factor_cut() != fgraph_cut || leaf_size<T>() != fgraph_leaf) {
      fgraph_cut = factor_cut();
      fgraph_leaf = leaf_size<T>();
      if (fgraph) cudaGraphExecDestroy(fgraph);
      fgraph = nullptr;
      fgraph_key = key;
      fgraph_runs = 0;
    }
    if (fgraph) {
      SAPB_CUDA(cudaGraphLaunch(fgraph, st));
      count_launch((int)fgraph_launches);
      g_lib_calls.fetch_add(fgraph_lib_calls, std::memory_order_relaxed);
    } else if (fgraph_runs >= 1 && !fgraph_failed && graph_enabled()) {
      const int64_t l0 = g_launches.load(), c0 = g_lib_calls.load();
      cudaGraph_t g = nullptr;
      bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        try {
          enqueue_factor(boost);
        } catch (...) {
          ok = false;
        }
        ok = (cudaStreamEndCapture(st, &g) == cudaSuccess) && ok && g;
      }
      if (ok) ok = cudaGraphInstantiate(&fgraph, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
      (void)cudaGetLastError();
      fgraph_launches = g_launches.load() - l0;
      fgraph_lib_calls = g_lib_calls.load() - c0;
      if (ok) {
        SAPB_CUDA(cudaGraphLaunch(fgraph, st));
      } else {
        fgraph = nullptr;
        fgraph_failed = true;  // run directly from now on
        enqueue_factor(boost);
      }
    } else {
      enqueue_factor(boost);
      fgraph_runs++;
    }
    int hf = 0;
    SAPB_CUDA(cudaMemcpyAsync(&hf, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    SAPB_CUDA(cudaStreamSynchronize(st));
    check_gemm();
    if (hf && !boost) throw Error(SAP_ZERO_PIVOTING, "Found a pivot equal to zero (partBandedLU).");
    make_half();
  }

  void enqueue_factor(bool boost) {
    flag.zero(st);
    BlockLU<T> lu;
    lu.h = h;
    lu.st = st;
    lu.batch = P;
    lu.boost = boost;
    lu.flag = flag.get();
    lu.cut = factor_cut();
    lanes(lu);
    lu.rws = std::max(1LL, BlockLU<T>::rec_ws(bs, lu.leaf));
    lu.rw = Rw.get();
    const Mat<T> D{Dw.get(), bs, BB}, Wm{Ww.get(), bs, BB};
    lu.W = Wm;
    for (int i = 0; i < nb; i++) {
      const Mat<T> Li = blk(Linv, nb, i), Ui = blk(Uinv, nb, i);
      {
        SAPB_PROF("wb_copy", st);
        lu.copy(Li, D, bs, bs);  // D_i (loaded into the L_ii^-1 slot)
        lu.fill(Li, bs, bs, T(0));
        lu.fill(Ui, bs, bs, T(0));
      }
      if (i > 0) {  // D_i -= L_{i,i-1} U_{i-1,i}: upper times lower
        SAPB_PROF("wb_schur", st);
        lu.prod_UL_acc(bs, T(-1), blk(Loff, nb - 1, i - 1), blk(Uoff, nb - 1, i - 1), D);
      }
      {
        SAPB_PROF("wb_rec", st);
        lu.rec(D, Li, Ui, bs);
      }
      if (i < nb - 1) {
        // U_{i,i+1} = L_ii^-1 E_i (lower times lower: E_i has no entries above
        // its diagonal) and, on the second lane, L_{i+1,i} = F_i U_ii^-1
        // (upper times upper); D is free again as the second lane's scratch
        SAPB_PROF("wb_offdiag", st);
        lu.fork();
        lu.prod_LL(bs, T(1), Li, blk(Uoff, nb - 1, i), Wm);
        lu.copy(Wm, blk(Uoff, nb - 1, i), bs, bs);
        lu.lane2([&] {
          lu.prod_UU(bs, T(1), blk(Loff, nb - 1, i), Ui, D);
          lu.copy(D, blk(Loff, nb - 1, i), bs, bs);
        });
        lu.join();
      }
    }
  }


  // tri: 0 full, 1 lower, 2 upper (see k_tgemv).  Grids with fewer than
  // about 2.5 CTAs per SM split the columns over gridDim.z CTAs.
  // Lanes (streams) for the block sweeps: each takes a contiguous share of
  // the partitions, so one lane's launch tails overlap the others'
  // streaming.  Each lane has its own column-split scratch.
  static constexpr int kMaxLanes = 4;
  DBuf<T> gws[kMaxLanes];          // column-split partial sums
  DBuf<unsigned> gctr[kMaxLanes];  // column-split arrival counters (zero between launches)
  cudaStream_t st2 = nullptr, st_more[kMaxLanes - 2] = {};
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_lane[kMaxLanes] = {};
  cudaStream_t lane_stream(int lane) const { return lane == 0 ? st : (lane == 1 ? st2 : st_more[lane - 2]); }
  // CTAs one GEMV launch aims at through its column split (about 2.5 of the
  // three resident CTAs per SM); SAPB_GEMV_CTAS overrides
  static int gemv_ctas() {
    const char* e = std::getenv("SAPB_GEMV_CTAS");
    return (e && std::atoi(e) > 0) ? std::atoi(e) : 370;
  }
  template <int V, typename MT = T>
  void gemv_launch(const MT* A, int ld, long long sA, const T* x, long long sx, const T* c, long long sc, T* y,
                   long long sy, int m, int nbatch, int mode, int tri, int lane, const T* cs = nullptr,
                   long long scs = 0) {
    cudaStream_t ls = lane_stream(lane);
    DBuf<T>& ws_ = gws[lane];
    DBuf<unsigned>& ct = gctr[lane];
    constexpr int R = tgemv_rows<T, V>();
    const int ntile = (m + R - 1) / R, pairs = (ntile + 1) / 2;
    const long long base = (long long)pairs * nbatch;
    const long long target = gemv_ctas();
    int S = (int)std::min<long long>(8, (target + base - 1) / base);
    S = std::max(1, std::min(S, m / 256));
    if (S > 1) {
      const size_t need = (size_t)nbatch * ntile * S * R, nctr = (size_t)nbatch * ntile;
      if (ws_.size() < need) ws_.alloc(need);
      if (ct.size() < nctr) {
        SAPB_CUDA(cudaStreamSynchronize(ls));
        ct.alloc(nctr);
        ct.zero(ls);
      }
    }
    // programmatic dependent launch (the kernel waits for its predecessor
    // on the device, see k_tgemv)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(pairs, nbatch, S);
    cfg.blockDim = dim3(kGemvWarps * 32);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ls;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SAPB_CUDA(cudaLaunchKernelEx(&cfg, k_tgemv<T, V, MT>, A, ld, sA, x, sx, c, sc, y, sy, m, mode, tri, ws_.get(),
                                 ct.get(), cs, scs));
    SAPB_LAUNCHED();
  }
  void gemv(const T* A, int ld, long long sA, const T* x, long long sx, const T* c, long long sc, T* y, long long sy,
            int m, int nbatch, int mode, int tri, int lane = 0) {
    constexpr int V = 16 / sizeof(T);  // 16-byte loads
    const bool vec = ld % V == 0 && sA % V == 0 && (reinterpret_cast<uintptr_t>(A) % 16) == 0;
    if (vec) gemv_launch<V>(A, ld, sA, x, sx, c, sc, y, sy, m, nbatch, mode, tri, lane);
    else gemv_launch<1>(A, ld, sA, x, sx, c, sc, y, sy, m, nbatch, mode, tri, lane);
  }
  // the same with an FP16 block-scaled matrix (column scales cs, batch stride scs)
  void gemv(const __half* A, const T* cs, long long scs, int ld, long long sA, const T* x, long long sx, const T* c,
            long long sc, T* y, long long sy, int m, int nbatch, int mode, int tri, int lane = 0) {
    if constexpr (sizeof(T) == 4) {
      const bool vec = ld % 8 == 0 && sA % 8 == 0 && (reinterpret_cast<uintptr_t>(A) % 16) == 0;
      if (vec) gemv_launch<8, __half>(A, ld, sA, x, sx, c, sc, y, sy, m, nbatch, mode, tri, lane, cs, scs);
      else gemv_launch<1, __half>(A, ld, sA, x, sx, c, sc, y, sy, m, nbatch, mode, tri, lane, cs, scs);
    } else {
      throw Error(SAP_ERR_INVALID_ARGUMENT, "FP16 block storage needs an FP32 preconditioner");
    }
  }

  // x <- A_p^-1 x for the padded block vectors of all partitions.  L_ii^-1
  // and U_{i,i+1} = L_ii^-1 E_i are lower triangular, U_ii^-1 and
  // L_{i+1,i} = F_i U_ii^-1 upper triangular (the band fits in one block).
  // Persistent sweeps (k_sweep, one cooperative launch per sweep): group
  // size G and column slices S per partition, scratch and barrier words.
  DBuf<T> pws;
  DBuf<unsigned> pctr, pbar;
  DBuf<int> perr;
  PinnedBuf<int> perr_h;
  template <int V, typename MT>
  bool sweep_persistent(T* x, const MT* Li, const MT* Ui, const MT* Lo, const MT* Uo, const T* cL, const T* cU,
                        const T* cLo, const T* cUo) {
    auto kern = k_sweep<T, V, MT>;
    int dev = 0, sms = 0, occ = 0, coop = 0;
    SAPB_CUDA(cudaGetDevice(&dev));
    SAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SAPB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    SAPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kGemvWarps * 32, 0));
    const int gmax = occ * sms / P;
    if (!coop || gmax < 1) return false;
    constexpr int R = tgemv_rows<T, V>();
    const int ntile = (bs + R - 1) / R, pairs = (ntile + 1) / 2;
    int S = 1, G = gmax;
    if (pairs <= gmax) {
      S = std::max(1, std::min({8, gmax / pairs, std::max(1, bs / 256)}));
      G = pairs * S;
    }
    pws.ensure((size_t)P * ntile * S * R);
    if (pctr.size() < (size_t)P * ntile) {
      pctr.alloc((size_t)P * ntile);
      pctr.zero(st);
    }
    if (pbar.size() < (size_t)2 * P) {
      pbar.alloc((size_t)2 * P);
      pbar.zero(st);
    }
    if (perr.size() == 0) {
      perr.alloc(1);
      perr.zero(st);
      *perr_h.reserve(1) = 0;
    }
    T* y = yv.get();
    T* t = tv.get();
    T* ws = pws.get();
    unsigned* ctr = pctr.get();
    unsigned* bar = pbar.get();
    int* err = perr.get();
    int nbv = nb, bsv = bs;
    long long BBv = BB, plenv = plen;
    // SAPB_TEST_BARRIER_STALL = 1: every group barrier waits for one CTA
    // more than exists, so that its bounded wait runs out and the error path
    // is taken (tests only)
    const char* se = std::getenv("SAPB_TEST_BARRIER_STALL");
    int stall = (se && std::atoi(se) == 1) ? 1 : 0;
    void* args[] = {(void*)&Li, (void*)&Ui, (void*)&Lo, (void*)&Uo, (void*)&cL, (void*)&cU, (void*)&cLo, (void*)&cUo,
                    (void*)&x, (void*)&y, (void*)&t, (void*)&nbv, (void*)&bsv, (void*)&BBv, (void*)&plenv, (void*)&G,
                    (void*)&S, (void*)&ws, (void*)&ctr, (void*)&bar, (void*)&err, (void*)&stall};
    SAPB_CUDA(cudaLaunchCooperativeKernel((const void*)kern, dim3((unsigned)(P * G)), dim3(kGemvWarps * 32), args, 0,
                                          st));
    count_launch();
    SAPB_CUDA(cudaMemcpyAsync(perr_h.get(), err, sizeof(int), cudaMemcpyDeviceToHost, st));
    return true;
  }
  // after the caller synchronised the stream: a barrier of a persistent
  // sweep that timed out is reported (and the barrier state reset)
  void check_device() {
    if (!perr_h.get() || *perr_h.get() == 0) return;
    *perr_h.get() = 0;
    perr.zero(st);
    pbar.zero(st);
    pctr.zero(st);
    SAPB_CUDA(cudaStreamSynchronize(st));
    throw Error(SAP_ERR_DEVICE_TIMEOUT, "a block-sweep barrier wait ran out of its iteration limit");
  }
  // One block sweep in schedule `mode`: 0 persistent (k_sweep), 1 / 2 / 4
  // lanes of per-step launches (fewer when a lane would get fewer than two
  // partitions).  False when the persistent launch is not possible.
  bool run_sweep(T* x, int mode) {
    if (mode == 0) {
      if (h16) {
        if constexpr (sizeof(T) == 4)
          return sweep_persistent<8, __half>(x, Lh.get(), Uh.get(), Loh.get(), Uoh.get(), csL.get(), csU.get(),
                                             csLo.get(), csUo.get());
        return false;
      }
      constexpr int V = 16 / sizeof(T);
      return bs % V == 0 && sweep_persistent<V, T>(x, Linv.get(), Uinv.get(), Loff.get(), Uoff.get(), nullptr,
                                                   nullptr, nullptr, nullptr);
    }
    int lanes = st2 ? mode : 1;
    while (lanes > 1 && P < 2 * lanes) lanes /= 2;
    if (lanes > 1) {
      SAPB_CUDA(cudaEventRecord(ev_fork, st));
      for (int l = 1; l < lanes; l++) SAPB_CUDA(cudaStreamWaitEvent(lane_stream(l), ev_fork, 0));
    }
    for (int lane = 0; lane < lanes; lane++) {
      const int p0 = (int)((long long)P * lane / lanes), p1 = (int)((long long)P * (lane + 1) / lanes);
      const long long vo = (long long)p0 * plen;
      solve_blocks_part(x + vo, yv.get() + vo, tv.get() + vo, p0, p1 - p0, lane);
    }
    for (int l = 1; l < lanes; l++) {
      SAPB_CUDA(cudaEventRecord(ev_lane[l], lane_stream(l)));
      SAPB_CUDA(cudaStreamWaitEvent(st, ev_lane[l], 0));
    }
    return true;
  }

  // Sweep schedule autotuner, keyed on the layout (P, block size, blocks per
  // partition, bytes per factor value): the first sweep of an unseen key
  // times the candidate schedules (persistent, 2 lanes, 4 lanes; best of
  // two runs each, CUDA events) on a copy of its right-hand side and keeps
  // the fastest for the process.  Measured on the 1M-row workload: the
  // persistent sweep for the FP16 copies (2.77 ms against 3.10 / 3.21 with 4
  // / 2 lanes), 2 lanes for FP32 / FP64 (3.90 / 7.05 ms against 3.97 / 7.29
  // persistent).  SAPB_SWEEP_PERSISTENT = 1 (or 0) and SAPB_SWEEP_LANES =
  // 1 / 2 / 4 fix the schedule instead.
  DBuf<T> tune_x;
  static std::map<std::tuple<int, int, int, int>, int>& tuned() {
    static std::map<std::tuple<int, int, int, int>, int> m;
    return m;
  }
  static int fixed_mode() {
    const char* pe = std::getenv("SAPB_SWEEP_PERSISTENT");
    const char* le = std::getenv("SAPB_SWEEP_LANES");
    int lanes = le ? std::atoi(le) : 0;
    if (lanes != 1 && lanes != 2 && lanes != 4) lanes = 0;
    if (pe && std::atoi(pe) != 0) return 0;
    if (pe || lanes) return lanes ? lanes : 2;
    return -1;
  }
  int tune_sweep(const T* x) {
    const size_t len = (size_t)P * plen;
    tune_x.ensure(len);
    cudaEvent_t a = nullptr, b = nullptr;
    SAPB_CUDA(cudaEventCreate(&a));
    SAPB_CUDA(cudaEventCreate(&b));
    int best = 2;
    float best_ms = 1e30f;
    for (int mode : {0, 2, 4}) {
      if (mode == 4 && P < 8) continue;
      float t = 1e30f;
      bool ok = true;
      for (int r = 0; r < 2 && ok; r++) {
        SAPB_CUDA(cudaMemcpyAsync(tune_x.get(), x, len * sizeof(T), cudaMemcpyDeviceToDevice, st));
        SAPB_CUDA(cudaEventRecord(a, st));
        ok = run_sweep(tune_x.get(), mode);
        SAPB_CUDA(cudaEventRecord(b, st));
        SAPB_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        SAPB_CUDA(cudaEventElapsedTime(&ms, a, b));
        if (ok) t = std::min(t, ms);
      }
      if (ok && t < best_ms) {
        best_ms = t;
        best = mode;
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    check_device();
    return best;
  }
  void solve_blocks(T* x) {
    int mode = fixed_mode();
    if (mode < 0) {
      const auto key = std::make_tuple(P, bs, nb, h16 ? 2 : (int)sizeof(T));
      auto it = tuned().find(key);
      if (it == tuned().end()) it = tuned().emplace(key, tune_sweep(x)).first;
      mode = it->second;
    }
    if (!run_sweep(x, mode)) run_sweep(x, 2);
  }

  // the block sweeps of partitions [p0, p0+np) on one lane
  void solve_blocks_part(T* x, T* y, T* t, int p0, int np, int lane) {
    if (h16) return solve_blocks_part_h16(x, y, t, p0, np, lane);
    const long long sv = plen;
    const long long od = (long long)p0 * nb * BB, oo = (long long)p0 * (nb - 1) * BB;
    for (int i = 0; i < nb; i++) {  // y_i = L_ii^-1 (x_i - L_{i,i-1} y_{i-1})
      const T* rhs = x + (long long)i * bs;
      if (i > 0) {
        gemv(Loff.get() + oo + (long long)(i - 1) * BB, bs, (long long)(nb - 1) * BB, y + (long long)(i - 1) * bs, sv,
             x + (long long)i * bs, sv, t, sv, bs, np, 1, 2, lane);
        rhs = t;
      }
      gemv(Linv.get() + od + (long long)i * BB, bs, (long long)nb * BB, rhs, sv, nullptr, 0, y + (long long)i * bs, sv,
           bs, np, 0, 1, lane);
    }
    for (int i = nb - 1; i >= 0; i--) {  // x_i = U_ii^-1 (y_i - U_{i,i+1} x_{i+1})
      const T* rhs = y + (long long)i * bs;
      if (i < nb - 1) {
        gemv(Uoff.get() + oo + (long long)i * BB, bs, (long long)(nb - 1) * BB, x + (long long)(i + 1) * bs, sv,
             y + (long long)i * bs, sv, t, sv, bs, np, 1, 1, lane);
        rhs = t;
      }
      gemv(Uinv.get() + od + (long long)i * BB, bs, (long long)nb * BB, rhs, sv, nullptr, 0, x + (long long)i * bs, sv,
           bs, np, 0, 2, lane);
    }
  }
  // the same sweeps over the FP16 copies
  void solve_blocks_part_h16(T* x, T* y, T* t, int p0, int np, int lane) {
    const long long sv = plen;
    const long long od = (long long)p0 * nb * BB, oo = (long long)p0 * (nb - 1) * BB;
    const long long cd = (long long)p0 * nb * bs, co = (long long)p0 * (nb - 1) * bs;
    const long long sd = (long long)nb * BB, so = (long long)(nb - 1) * BB;
    const long long csd = (long long)nb * bs, cso = (long long)(nb - 1) * bs;
    for (int i = 0; i < nb; i++) {
      const T* rhs = x + (long long)i * bs;
      if (i > 0) {
        gemv(Loh.get() + oo + (long long)(i - 1) * BB, csLo.get() + co + (long long)(i - 1) * bs, cso, bs, so,
             y + (long long)(i - 1) * bs, sv, x + (long long)i * bs, sv, t, sv, bs, np, 1, 2, lane);
        rhs = t;
      }
      gemv(Lh.get() + od + (long long)i * BB, csL.get() + cd + (long long)i * bs, csd, bs, sd, rhs, sv, nullptr, 0,
           y + (long long)i * bs, sv, bs, np, 0, 1, lane);
    }
    for (int i = nb - 1; i >= 0; i--) {
      const T* rhs = y + (long long)i * bs;
      if (i < nb - 1) {
        gemv(Uoh.get() + oo + (long long)i * BB, csUo.get() + co + (long long)i * bs, cso, bs, so,
             x + (long long)(i + 1) * bs, sv, y + (long long)i * bs, sv, t, sv, bs, np, 1, 1, lane);
        rhs = t;
      }
      gemv(Uh.get() + od + (long long)i * BB, csU.get() + cd + (long long)i * bs, csd, bs, sd, rhs, sv, nullptr, 0,
           x + (long long)i * bs, sv, bs, np, 0, 2, lane);
    }
  }


  // Interface positions inside the partitions' block vectors: pos[t][k] for
  // the bottom (which 0, partition t) or top (which 1, partition t+1) unknowns.
  std::vector<int> iface_pos(const std::vector<int>& iface, int which) const {
    const int nI = P - 1;
    std::vector<int> pos((size_t)nI * K);
    for (int t = 0; t < nI; t++)
      for (int k = 0; k < K; k++) {
        const int q = iface[(size_t)t * 2 * K + (size_t)which * K + k] - pstart_h[t + which];
        if (q < 0 || q >= psize_h[t + which]) throw Error(SAP_ERR_INVALID_ARGUMENT, "interface row outside its partition");
        pos[(size_t)t * K + k] = q;
      }
    return pos;
  }

  // Spike tips of every interface t (column-major K x K):
  //   V_t = rows at the bottom interface unknowns of A_t^-1 [.. B_t ..],
  //   W_t = rows at the top interface unknowns of A_{t+1}^-1 [.. C_t ..],
  // by block solves whose right-hand sides are the coupling blocks' nonzero
  // columns, batched over the interfaces (slabs of columns bound the memory).
  // offd (device): row-major coupling blocks, B_t at 2t, C_t at 2t+1;
  // iface: [P-1][2K] band rows, bottom unknowns of partition t, then top
  // unknowns of partition t+1.
  void spikes(const T* offd, const std::vector<int>& iface, int K_) {
    K = K_;
    constexpr int V = 16 / sizeof(T);
    ldK = (K + V - 1) / V * V;
    sK = (long long)ldK * K;
    spike = true;
    const int nI = P - 1;
    Vc.alloc((size_t)nI * sK);
    Wc.alloc((size_t)nI * sK);
    Vc.zero(st);
    Wc.zero(st);
    std::vector<int> nzh((size_t)2 * nI * K);
    {
      nz_d.ensure(nzh.size());
      k_nz_cols<T><<<dim3(grid1d(K, 256, 64), 2 * nI), 256, 0, st>>>(offd, K, nz_d.get());
      SAPB_LAUNCHED();
      SAPB_CUDA(cudaMemcpyAsync(nzh.data(), nz_d.get(), nzh.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
      SAPB_CUDA(cudaStreamSynchronize(st));
    }
    // the X slab holds nI * plen * cs values
    const double budget = 8.0e9;
    const int cs_max = (int)std::max<double>(32.0, std::min<double>(K, budget / ((double)nI * plen * sizeof(T))));
    for (int which = 0; which < 2; which++) {
      const std::vector<int> pos = iface_pos(iface, which);
      int ncol = 0, minpos = (int)plen;
      std::vector<int> cnt(nI, 0);
      for (int t = 0; t < nI; t++) {
        for (int c = 0; c < K; c++) cnt[t] += nzh[(size_t)(2 * t + which) * K + c];
        ncol = std::max(ncol, cnt[t]);
        for (int k = 0; k < K; k++) minpos = std::min(minpos, pos[(size_t)t * K + k]);
      }
      if (ncol == 0) continue;
      std::vector<int> cols((size_t)nI * ncol, -1);
      for (int t = 0; t < nI; t++) {
        int j = 0;
        for (int c = 0; c < K; c++)
          if (nzh[(size_t)(2 * t + which) * K + c]) cols[(size_t)t * ncol + j++] = c;
      }
      // (buffers grow only: the two sides and repeated setups reuse them)
      DBuf<int>& cols_d = spk_cols[which];
      DBuf<int>& pos_d = spk_pos[which];
      cols_d.put(cols, st);
      pos_d.put(pos, st);
      const int cs = std::min(ncol, cs_max);
      const long long sX = plen * cs;
      X.ensure((size_t)nI * sX);
      Wt.ensure((size_t)nI * bs * cs);
      BlockLU<T> ops;
      ops.h = h;
      ops.st = st;
      ops.batch = nI;
      ops.cut = spike_cut();
      ops.tc = tc_on();
      ops.gerr = gemm_err.get();
      const Mat<T> Wm{Wt.get(), bs, (long long)bs * cs};
      const int ib0 = std::max(0, minpos) / bs;
      auto Xb = [&](int i) { return Mat<T>{X.get() + (long long)i * bs, (int)plen, sX}; };
      // factor blocks of partition t + which for interface t
      auto Fk = [&](DBuf<T>& a, int per, int i) {
        return Mat<T>{a.get() + (long long)which * per * BB + (long long)i * BB, bs, (long long)per * BB};
      };
      const int kt = std::min(1024, ((K + 31) / 32) * 32);
      for (int j0 = 0; j0 < ncol; j0 += cs) {
        const int w = std::min(cs, ncol - j0);
        // only block rows ib0.. of each column are written or read below
        SAPB_CUDA(cudaMemset2DAsync(X.get() + (long long)ib0 * bs, (size_t)plen * sizeof(T), 0,
                                    (size_t)(plen - (long long)ib0 * bs) * sizeof(T), (size_t)nI * cs, st));
        k_spike_rhs<T><<<dim3(w, nI), kt, 0, st>>>(offd, which, K, cols_d.get(), ncol, j0, pos_d.get(), X.get(), sX,
                                                    plen);
        SAPB_LAUNCHED();
        // forward with L_{i,i-1} (upper) and L_ii^-1 (lower), backward with
        // U_{i,i+1} (lower) and U_ii^-1 (upper)
        for (int i = ib0; i < nb; i++) {
          if (i > ib0) ops.prod_UF(bs, w, T(-1), Fk(Loff, nb - 1, i - 1), Xb(i - 1), T(1), Xb(i));
          ops.prod_LF(bs, w, T(1), Fk(Linv, nb, i), Xb(i), T(0), Wm);
          ops.copy(Wm, Xb(i), bs, w);
        }
        for (int i = nb - 1; i >= ib0; i--) {
          if (i < nb - 1) ops.prod_LF(bs, w, T(-1), Fk(Uoff, nb - 1, i), Xb(i + 1), T(1), Xb(i));
          ops.prod_UF(bs, w, T(1), Fk(Uinv, nb, i), Xb(i), T(0), Wm);
          ops.copy(Wm, Xb(i), bs, w);
        }
        k_spike_tips<T><<<dim3(w, nI), kt, 0, st>>>(X.get(), sX, plen, cols_d.get(), ncol, j0, pos_d.get(), K, ldK,
                                                     sK, which ? Wc.get() : Vc.get());
        SAPB_LAUNCHED();
      }
      SAPB_CUDA(cudaStreamSynchronize(st));
    }
    check_gemm();
  }

  // S_t = I - W_t V_t, factored with its triangular inverses (boosted only
  // when `boost`); coupling blocks kept column-major for the apply.
  void reduced(const T* offd, const std::vector<int>& iface, bool boost) {
    math_mode(tf32 && reduced_tf32());
    const int nI = P - 1;
    Bc.alloc((size_t)nI * sK);
    Cc.alloc((size_t)nI * sK);
    Bc.zero(st);
    Cc.zero(st);
    const dim3 tg((K + 31) / 32, (K + 31) / 32, nI);
    k_couple_colmajor<T><<<tg, dim3(32, 8), 0, st>>>(offd, 0, K, ldK, sK, Bc.get());
    SAPB_LAUNCHED();
    k_couple_colmajor<T><<<tg, dim3(32, 8), 0, st>>>(offd, 1, K, ldK, sK, Cc.get());
    SAPB_LAUNCHED();
    S.alloc((size_t)nI * sK);
    Ws.alloc((size_t)nI * sK);
    sflag.alloc(1);
    sflag.zero(st);
    SLi.alloc((size_t)nI * sK);
    SUi.alloc((size_t)nI * sK);
    SLi.zero(st);
    SUi.zero(st);
    k_identity<T><<<dim3(grid1d(sK, 256, 4096), nI), 256, 0, st>>>(S.get(), K, ldK, sK);
    SAPB_LAUNCHED();
    BlockLU<T> lu;
    lu.h = h;
    lu.st = st;
    lu.batch = nI;
    lu.boost = boost;
    lu.flag = sflag.get();
    lu.W = Mat<T>{Ws.get(), ldK, sK};
    lanes(lu);
    lu.tc = tc_on() && reduced_tf32();
    lu.rws = std::max(1LL, BlockLU<T>::rec_ws(K, lu.leaf));
    Rs.alloc((size_t)nI * lu.rws);
    lu.rw = Rs.get();
    const Mat<T> Sm{S.get(), ldK, sK};
    lu.gemm(K, K, K, T(-1), Mat<T>{Wc.get(), ldK, sK}, Mat<T>{Vc.get(), ldK, sK}, T(1), Sm);
    lu.rec(Sm, Mat<T>{SLi.get(), ldK, sK}, Mat<T>{SUi.get(), ldK, sK}, K);
    std::vector<long long> pos((size_t)nI * 2 * K), rows((size_t)nI * 2 * K);
    for (int which = 0; which < 2; which++) {
      const std::vector<int> q = iface_pos(iface, which);
      for (int t = 0; t < nI; t++)
        for (int k = 0; k < K; k++) {
          const size_t e = (size_t)t * 2 * K + (size_t)which * K + k;
          pos[e] = (t + which) * plen + q[(size_t)t * K + k];
          rows[e] = iface[e];
        }
    }
    ipos.upload(pos, st);
    irow.upload(rows, st);
    xbt.alloc((size_t)nI * 2 * K);
    fbt.alloc((size_t)nI * 2 * K);
    t1.alloc((size_t)nI * K);
    t2.alloc((size_t)nI * K);
    SAPB_CUDA(cudaStreamSynchronize(st));
    check_gemm();
  }

  // Reduced solve and purification: x holds A_p^-1 f (block layout), F the
  // band-order right-hand side; F's interface rows get f -= offdiag * z.
  void reduced_apply(const T* x, T* F) {
    const int nI = P - 1;
    const long long m = (long long)nI * 2 * K, s2 = 2LL * K;
    k_gather_idx<T><<<grid1d(m), 256, 0, st>>>(x, ipos.get(), m, xbt.get());
    SAPB_LAUNCHED();
    k_gather_idx<T><<<grid1d(m), 256, 0, st>>>(F, irow.get(), m, fbt.get());
    SAPB_LAUNCHED();
    T* xb = xbt.get();
    T* xt = xbt.get() + K;
    T* fb = fbt.get();
    T* ft = fbt.get() + K;
    gemv(Wc.get(), ldK, sK, xb, s2, xt, s2, t1.get(), K, K, nI, 1, 0);            // t1 = xt - W xb
    gemv(SLi.get(), ldK, sK, t1.get(), K, nullptr, 0, t2.get(), K, K, nI, 0, 1);  // t2 = L_S^-1 t1
    gemv(SUi.get(), ldK, sK, t2.get(), K, nullptr, 0, t1.get(), K, K, nI, 0, 2);  // z2 = U_S^-1 t2
    gemv(Vc.get(), ldK, sK, t1.get(), K, xb, s2, t2.get(), K, K, nI, 1, 0);       // z1 = xb - V z2
    gemv(Bc.get(), ldK, sK, t1.get(), K, fb, s2, fb, s2, K, nI, 1, 0);            // f_b -= B z2
    gemv(Cc.get(), ldK, sK, t2.get(), K, ft, s2, ft, s2, K, nI, 1, 0);            // f_t -= C z1
    k_scatter_idx<T><<<grid1d(m), 256, 0, st>>>(irow.get(), fbt.get(), m, F);
    SAPB_LAUNCHED();
  }

  // z = M^-1 v: leftTrans gather (gin/sin), partition solves, reduced
  // correction, partition solves, rightTrans scatter (sout/cout).  The
  // permutation arguments are null for a matrix used in its own order.
  void apply(const double* v, double* z, const int* gin, const T* sin, const int* sout, const T* cout) {
    wait_half();
    const dim3 gb(grid1d(plen, 256, 1024), P);
    k_wb_in<T><<<grid1d(n), 256, 0, st>>>(v, gin, sin, Fb.get(), n);
    SAPB_LAUNCHED();
    k_wb_to_blocks<T><<<gb, 256, 0, st>>>(Fb.get(), xv.get(), pstart_d.get(), psize_d.get(), plen);
    SAPB_LAUNCHED();
    {
      SAPB_PROF("block_sweep", st);
      solve_blocks(xv.get());
    }
    if (spike) {
      {
        SAPB_PROF("reduced_apply", st);
        reduced_apply(xv.get(), Fb.get());
      }
      k_wb_to_blocks<T><<<gb, 256, 0, st>>>(Fb.get(), xv.get(), pstart_d.get(), psize_d.get(), plen);
      SAPB_LAUNCHED();
      SAPB_PROF("block_sweep", st);
      solve_blocks(xv.get());
    }
    k_wb_out<T><<<grid1d(n), 256, 0, st>>>(xv.get(), rowpart_d.get(), pstart_d.get(), plen, sout, cout, z, n);
    SAPB_LAUNCHED();
  }
};

}  // namespace sapb
