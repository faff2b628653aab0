/*
 * sap_b200.h — C ABI of the B200-native SPIKE-preconditioned Krylov solver.
 *
 * The reference (spikegpu/SaPLibrary) exposes this path only as C++
 * templates; every entry point below names the reference interface it
 * replaces (file:line, relative to the reference project root).  Plain
 * pointers and sizes only: no CUDA, torch or C++ types cross the boundary.
 *
 * Conventions
 *  - Every function returns an int status: 0 on success, one of the
 *    sap::system_error::Reason values (sap/exception.h:16-23) for the
 *    reference's own failures, or one of the SAP_ERR_* codes below.
 *  - `memspace` arguments say where a caller buffer lives:
 *    SAP_HOST (pageable or pinned host memory) or SAP_DEVICE (memory of the
 *    current CUDA device).
 *  - All device work of one solver runs on that solver's own CUDA stream;
 *    a call returns after its results are complete (setup, update, solve),
 *    except the *_async device-pointer helpers, which only enqueue.
 *  - Handles are not re-entrant (the reference Solver is not either:
 *    sap/solver.h:153-225 keeps mutable work vectors).
 */
#ifndef SAP_B200_H
#define SAP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  SAP_OK = 0,
  /* sap::system_error::Reason (sap/exception.h:16-23) */
  SAP_ZERO_PIVOTING = -1,
  SAP_NEGATIVE_DB_WEIGHT = -2,
  SAP_ILLEGAL_UPDATE = -3,
  SAP_ILLEGAL_SOLVE = -4,
  SAP_MATRIX_SINGULAR = -5,
  /* library errors with no reference counterpart */
  SAP_ERR_INVALID_ARGUMENT = -100,
  SAP_ERR_CUDA = -101,
  SAP_ERR_OUT_OF_MEMORY = -102,
  SAP_ERR_UNSUPPORTED = -103,
  SAP_ERR_DEVICE_TIMEOUT = -104
};

enum { SAP_HOST = 0, SAP_DEVICE = 1 };

/* KrylovSolverType (sap/common.h:71-82); CUSP solvers are not provided. */
enum {
  SAP_BICGSTAB_C = 0, SAP_GMRES_C = 1, SAP_CG_C = 2, SAP_CR_C = 3,
  SAP_BICGSTAB1 = 4, SAP_BICGSTAB2 = 5, SAP_BICGSTAB = 6, SAP_MINRES = 7,
  /* Extension (not in the reference): flexible right-preconditioned
   * GMRES(50) with FP64 Arnoldi, which tolerates a preconditioner that
   * changes between applies (FP32 / TF32 factors) and so reaches FP64
   * tolerances without refinement restarts. */
  SAP_FGMRES = 8
};
/* FactorizationMethod (sap/common.h:86-89) */
enum { SAP_LU_UL = 0, SAP_LU_ONLY = 1 };
/* PreconditionerType (sap/common.h:94-98) */
enum { SAP_PRECOND_SPIKE = 0, SAP_PRECOND_BLOCK = 1, SAP_PRECOND_NONE = 2 };
/* Preconditioner value type: the Solver's PrecValueType template argument
 * (sap/solver.h:153). */
enum { SAP_PREC_FLOAT = 0, SAP_PREC_DOUBLE = 1, SAP_PREC_TF32 = 2, SAP_PREC_TF32_F16 = 3 };

/* sap::Options (sap/solver.h:52-81); same fields, same defaults
 * (sap/solver.h:233-256).  Booleans are ints (0/1). */
typedef struct sap_options {
  int solverType;
  int maxNumIterations;
  double relTol;
  double absTol;
  int testDB;
  int isSPD;
  int saveMem;
  int performReorder;
  int performDB;
  int dbFirstStageOnly;
  int applyScaling;
  int maxBandwidth;
  int gpuCount;
  double dropOffFraction;
  int factMethod;
  int precondType;
  int safeFactorization;
  int variableBandwidth;
  int trackReordering;
  int useBCR;
  int ilu_level;
  /* Extension (not in the reference): when > 0, solve() runs up to this many
   * FP64 iterative-refinement sweeps r = b - A x, A d = r by BiCGStab(L)
   * (stopping at the global tolerance, on stagnation or at the iteration
   * budget), x += d.  0 (the default) runs the reference's single solve. */
  int refinementSweeps;
} sap_options;

/* sap::Stats (sap/solver.h:89-140); times in milliseconds as in the
 * reference's timers (sap/timer.h). */
typedef struct sap_stats {
  double timeSetup, timeUpdate, timeSolve;
  double time_DB, time_DB_pre, time_DB_first, time_DB_second, time_DB_post;
  double d_p1, d_p1_ori, diag_dom, diag_dom_ori;
  double time_reorder, time_dropOff, time_cpu_assemble, time_transfer;
  double time_toBanded, time_offDiags, time_bandLU, time_bandUL;
  double time_fullLU, time_assembly, time_shuffle;
  int bandwidthReorder, bandwidthDB, bandwidth;
  double nuKf, flops_LU;
  int numPartitions;
  double actualDropOff;
  float numIterations;
  double rhsNorm, residualNorm, relResidualNorm;
  int actual_nnz;
} sap_stats;

typedef struct sap_solver sap_solver;   /* sap::Solver<Array,PrecValueType> */
typedef struct sap_banded sap_banded;   /* sap::BandedMatrix<Array> */
typedef struct sap_csr sap_csr;         /* cusp::csr_matrix<int,double,device> */
typedef struct sap_spmv sap_spmv;       /* SpMV functor (MVBanded / SpmvCusp) */

/* ---- errors ------------------------------------------------------------- */
/* Message of the last failure on the calling thread (what() of the
 * reference's sap::system_error, or the CUDA error string). */
const char* sap_last_error(void);

/* ---- options ------------------------------------------------------------ */
/* Options::Options() (sap/solver.h:233-256). */
int sap_options_default(sap_options* opts);

/* ---- matrices ----------------------------------------------------------- */
/* BandedMatrix(n, k, d) (sap/banded_matrix.h:59-95) from caller data: a
 * row-major band of n*(2k+1) doubles, element (i,j) at i*(2k+1)+k+(j-i).
 * The data is copied to the device. */
int sap_banded_create(int n, int k, const double* band_rowmajor, int memspace,
                      sap_banded** out);
/* BandedMatrix(n, k, d) generated in place (sap/banded_matrix.h:59-95).
 * dist: 0 = uniform[-10,10] from the C library rand() seeded with `seed`
 * (the reference generator), 1 = uniform[-1,1], 2 = standard normal; the
 * diagonal is d * (sum of |off-diagonals| of the row).  dists 1 and 2 use a
 * counter-based generator, identical for any thread count. */
int sap_banded_generate(int n, int k, double d, int dist, uint64_t seed, sap_banded** out);
/* The generator of sap_banded_generate run on the host into `out`
 * (n*(2k+1) doubles, row-major); needs no GPU. */
int sap_generate_band_host(int n, int k, double d, int dist, uint64_t seed, double* out);
/* Copy the row-major band back (host or device destination). */
int sap_banded_copy_out(const sap_banded* A, double* dst, int memspace);
int sap_banded_info(const sap_banded* A, int* n, int* k);
int sap_banded_destroy(sap_banded* A);

/* CSR matrix (int32 indices, FP64 values), copied to the device; the
 * reference's cusp::csr_matrix<int,double,device_memory>. */
int sap_csr_create(int n, int nnz, const int* row_offsets, const int* column_indices,
                   const double* values, int memspace, sap_csr** out);
int sap_csr_info(const sap_csr* A, int* n, int* nnz);
int sap_csr_destroy(sap_csr* A);

/* ---- SpMV functors (sap/spmv.h) ------------------------------------------ */
/* MVBanded(A) (sap/spmv.h:27-74): y = A x on the row-major FP64 band. */
int sap_spmv_banded_create(const sap_banded* A, sap_spmv** out);
/* SpmvCusp(A) (sap/spmv.h:83-129): y = A x, FP64 CSR. */
int sap_spmv_csr_create(const sap_csr* A, sap_spmv** out);
/* A user operator: fn(ctx, x, y, stream) computes y = A x on device
 * pointers, enqueued on `stream` (a cudaStream_t). */
typedef void (*sap_spmv_fn)(void* ctx, const double* x, double* y, void* stream);
int sap_spmv_callback_create(int n, sap_spmv_fn fn, void* ctx, sap_spmv** out);
/* operator()(v, Av) (sap/spmv.h:39-56, 110-121); device pointers. */
int sap_spmv_apply(sap_spmv* op, const double* x, double* y);
int sap_spmv_destroy(sap_spmv* op);

/* ---- BLAS-1 ------------------------------------------------------------------ */
/* nq <= 4 dot products out[q] = sum_i x[q][i] * y[q][i] of FP64 device
 * vectors in one pass: the fused form of the cusp::blas::dotc calls of the
 * Krylov monitor (sap/bicgstab2.h:98-300).  `out` is a device array of nq
 * doubles; the work is enqueued on `stream` (a cudaStream_t, NULL for the
 * legacy default stream) and the call returns without waiting.  Block partial
 * sums live in scratch allocated and freed on the stream by each call. */
int sap_blas_dots(int n, int nq, const double* const* x, const double* const* y, double* out, void* stream);
/* The same dot products with no allocation of any kind, for callers that
 * cannot allocate device memory where they need the reduction (code running
 * under another framework's caching allocator that owns the free memory,
 * applications that budget GPU memory once at start-up, loops in which a
 * cudaMalloc/cudaFree pair would synchronise the device).  No counterpart in
 * the reference.  The block partial sums live in a fixed 64 KB scratch array
 * compiled into the library, held by every GPU that loads it until exit;
 * n is limited to 16,777,216 (larger n returns SAP_ERR_INVALID_ARGUMENT).
 * The first call on a device looks up the scratch's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls on one device share its scratch,
 * which keeps the last call's contents (the completion counter is cleared by
 * each call): calls that overlap on the same GPU, for example on two
 * streams, race on it and must be serialised by the caller. */
int sap_blas_dots_noalloc(int n, int nq, const double* const* x, const double* const* y, double* out,
                          void* stream);

/* ---- tensor-core GEMM (no reference counterpart) ----------------------------
 * The batched product the wide-band block factorization, its spike slabs
 * and reduced systems run on in the TF32 forms, exposed for tests and
 * measurement: C_b = alpha A_b B_b + beta C_b for b < batch, column-major
 * FP32 device matrices (A m x k, B k x n, C m x n; leading dimensions lda,
 * ldb, ldc and batch strides sA, sB, sC in elements), TF32 inputs (rounded
 * to nearest) and FP32 accumulation on the sm_100 tensor cores (tcgen05,
 * operands staged by TMA).  A and B must be 16-byte aligned with lda, ldb,
 * sA, sB multiples of 4 (else SAP_ERR_UNSUPPORTED, nothing launched).  The
 * call enqueues on `stream` and waits for it; SAP_ERR_DEVICE_TIMEOUT if a
 * bounded wait inside the kernel ran out. */
int sap_tc_gemm_batched(int m, int n, int k, float alpha, const float* A, int lda, long long sA, const float* B,
                        int ldb, long long sB, float beta, float* C, int ldc, long long sC, int batch, void* stream);

/* ---- solver --------------------------------------------------------------- */
/* Solver(numPartitions, opts) (sap/solver.h:157-158, 268-297).  prec_dtype
 * is the preconditioner's PrecValueType: SAP_PREC_FLOAT or SAP_PREC_DOUBLE,
 * or SAP_PREC_TF32 (FP32 storage whose wide-band block products run on the
 * tensor cores in TF32 with FP32 accumulation; narrow bands as FP32), or
 * SAP_PREC_TF32_F16 (as SAP_PREC_TF32, and the wide-band block sweeps of the
 * apply read FP16 copies of the factor blocks scaled by a power of two per
 * column: half the bytes; extensions, no reference counterpart). */
int sap_solver_create(int num_partitions, const sap_options* opts, int prec_dtype,
                      sap_solver** out);
int sap_solver_destroy(sap_solver* s);

/* Solver::setup(A) (sap/solver.h:171, 339-404) for a BandedMatrix. */
int sap_solver_setup_banded(sap_solver* s, const sap_banded* A);
/* Solver::setup(A) for a CSR matrix (reordering per opts.performReorder). */
int sap_solver_setup_csr(sap_solver* s, const sap_csr* A);

/* Solver::update(entries) (sap/solver.h:174, 421-462): `entries` are the
 * nnz new CSR values in the pattern given to setup.  *accepted is 0 when
 * nnz differs from the setup matrix (the reference returns false). */
int sap_solver_update(sap_solver* s, const double* entries, int64_t nnz, int memspace,
                      int* accepted);

/* Solver::solve(spmv, b, x) (sap/solver.h:177-179, 477-562).  b and x live
 * in `memspace`; x is the initial guess on entry and the solution on exit.
 * *converged receives the reference's bool return value. */
int sap_solver_solve(sap_solver* s, sap_spmv* spmv, const double* b, double* x, int memspace,
                     int* converged);

/* Precond::operator()(v, z) (sap/precond.h:1370-1386): z = M^{-1} v on
 * device pointers of length n. */
int sap_precond_apply(sap_solver* s, const double* v, double* z);

/* Solver::getStats() (sap/solver.h:182). */
int sap_solver_get_stats(const sap_solver* s, sap_stats* out);
/* getMonitorCode / getMonitorMessage (sap/solver.h:183-194). */
int sap_solver_get_monitor(const sap_solver* s, int* code, const char** message);
/* Number of rows, the effective half-bandwidth and partition count after
 * setup (Precond::getBandwidth / getNumPartitions, sap/precond.h:152-157). */
int sap_solver_info(const sap_solver* s, int* n, int* k, int* num_partitions);
/* Reordering results of a CSR setup with reordering, as int arrays:
 * which = 0: DB row permutation (row i of A goes to row out[i]);
 * 1: composed row permutation, input row -> band row (Precond::m_optPerm
 *    after composition, sap/precond.h:2071-2097);
 * 2: composed column order, band column -> input column (m_optReordering);
 * 3: first_rows of the second-level reordering (graph.h:991-1007);
 * 4: per-partition half-bandwidths K_p (m_ks_host).
 * With out == NULL only *count is set. */
int sap_solver_get_reorder(const sap_solver* s, int which, int* out, int64_t* count);

/* The host reordering of a CSR setup on its own, without a device: the
 * matrix converted to the preconditioner type (SAP_PREC_FLOAT or
 * SAP_PREC_DOUBLE) with explicit zeros removed (precond.h:1667-1713), DB
 * matching and scaling with edge weights log(rowmax / |a|) computed on the
 * host (graph.h:1214-1361, 1875-2173), RCM (graph.h:1371-1584), drop-off
 * (graph.h:598-747), coupling split and second-level reordering
 * (graph.h:756-1008), variable half-bandwidths (graph.h:1093-1206) and the
 * composed permutations (precond.h:2071-2097), as a setup with
 * num_partitions and opts runs them (Graph::reorder and
 * transformToBandedMatrix's host part).  Outputs (NULL to skip): db_row_perm
 * and final_pos / final_order (n each, the arrays 0-2 of
 * sap_solver_get_reorder), first_rows (P-1, variable band only) and part_k
 * (P; K in every partition for a constant band), P <= num_partitions.  threads > 0 sets the host threads for this call (the
 * outputs do not depend on it).  Errors: SAP_ERR_INVALID_ARGUMENT, the DB's
 * SAP_MATRIX_SINGULAR / SAP_NEGATIVE_DB_WEIGHT.  Extension, no reference
 * counterpart as a separate call. */
typedef struct sap_reorder_info {
  int K, P, k_db, k_reorder, var_band;
  double drop_actual;
} sap_reorder_info;
int sap_reorder_host(int n, int nnz, const int* row_offsets, const int* column_indices, const double* values,
                     int num_partitions, const sap_options* opts, int prec_dtype, int threads,
                     sap_reorder_info* info, int* db_row_perm, int* final_pos, int* final_order, int* first_rows,
                     int* part_k);
/* Wall time (ms) of the stages of the calling thread's last successful
 * sap_reorder_host, in order ("db", "rcm", "drop_off", then for a variable
 * band "coupling", "second_level", "assemble", and "compose"): *count is
 * set to their number, and up to cap of them are written to names (static
 * strings) and ms (either may be NULL).  Extension, no reference
 * counterpart (the reference's Stats hold timeDB, timeReorder and
 * timeDropoff for a setup). */
int sap_reorder_host_stages(int cap, const char** names, double* ms, int* count);
/* The cudaStream_t all device work of this solver is enqueued on. */
void* sap_solver_stream(const sap_solver* s);
/* Layout of the wide-band block path after setup: the block size and the
 * number of blocks per partition (both 0 when the narrow band kernels are
 * used), and the bytes of one factor value read by the apply's sweeps (8, 4,
 * or 2 for the FP16 copies of SAP_PREC_TF32_F16). */
int sap_solver_block_layout(const sap_solver* s, int* block_size, int* blocks_per_partition, int* value_bytes);
/* Number of this library's own kernels enqueued since load (all handles). */
int64_t sap_kernel_launch_count(void);
/* Number of cuBLAS calls (batched GEMMs of the wide-band path) since load. */
int64_t sap_library_call_count(void);
/* Live kernel timing with CUDA events on the launching stream: while a
 * kernel name is selected, every launch of that kernel is bracketed by an
 * event pair; sap_profile_read returns the summed duration (ms) and the
 * number of launches since the selection (NULL or "" switches it off). */
int sap_profile_select(const char* kernel_name);
int sap_profile_read(double* total_ms, int64_t* launches);

/* ---- batched solve (no counterpart in the reference) -----------------------
 * Solves m independent banded systems A_i x_i = b_i (row-major bands of
 * n_i x (2 k_i + 1) values, host arrays) with the options' Krylov method and
 * preconditioner type.  Systems of equal half-bandwidth are solved together
 * as one block-diagonal system, every system's rows scaled by 1/||b_i||, to
 * the absolute residual opts->relTol, which gives each system
 * ||b_i - A_i x_i|| <= relTol ||b_i|| (opts->absTol is not used).  x_i are
 * the initial guesses' storage (overwritten; the solve starts from zero).
 * results[i]: the system's relative residual, the iterations of its stack
 * and whether it met relTol; seconds: wall time of the whole batch. */
typedef struct sap_batch_result {
  double rel_residual;
  float iterations;
  int converged;
} sap_batch_result;
int sap_batch_banded_solve(int m, const int* n, const int* k, const double* const* bands, const double* const* b,
                           double* const* x, int num_partitions, const sap_options* opts, int prec_dtype,
                           sap_batch_result* results, double* seconds);

/* ---- learned solver settings (no counterpart in the reference) -------------
 * A multilayer perceptron in -> h1 -> h2 -> out (ReLU hidden layers, softmax
 * output) mapping matrix features to a choice of solver settings, trained and
 * evaluated on the GPU by this library's kernels (FP32, deterministic).
 * Parameters are one flat float array: W1 [h1][in], b1, W2 [h2][h1], b2,
 * W3 [out][h2], b3.  Features, labels and outputs are host arrays. */
typedef struct sap_mlp sap_mlp;
int sap_mlp_create(int in, int h1, int h2, int out, uint64_t seed, sap_mlp** mlp);
int sap_mlp_destroy(sap_mlp* mlp);
int sap_mlp_num_params(const sap_mlp* mlp);
int sap_mlp_get_params(sap_mlp* mlp, float* params);
int sap_mlp_set_params(sap_mlp* mlp, const float* params);
/* logits[batch][out] of features x[batch][in] */
int sap_mlp_forward(sap_mlp* mlp, const float* x, int batch, float* logits);
/* mean softmax cross-entropy over the batch and its gradient (flat layout) */
int sap_mlp_gradients(sap_mlp* mlp, const float* x, const int* labels, int batch, float* grads, float* loss);
/* `epochs` full-batch Adam steps (beta 0.9 / 0.999); final mean loss */
int sap_mlp_train(sap_mlp* mlp, const float* x, const int* labels, int batch, int epochs, float lr, float* loss);
const char* sap_mlp_last_error(void);

/* ---- Matrix Market input ---------------------------------------------------
 * Replaces cusp::io::read_matrix_market_file of the reference drivers
 * (examples/driver_mm.cu).  Matrices: coordinate real / integer / pattern,
 * general / symmetric / skew-symmetric, returned as CSR (rows and columns
 * sorted, duplicates summed).  Call once with row_offsets / col_indices /
 * values NULL to get the sizes, then again with arrays of n_rows + 1 and nnz
 * elements.  Vectors: array (one column) or coordinate; call with values
 * NULL for the length.  Errors return SAP_ERR_INVALID_ARGUMENT with the
 * reason in sap_mm_last_error(). */
int sap_mm_read_csr(const char* path, int* n_rows, int* n_cols, int64_t* nnz, int* row_offsets, int* col_indices,
                    double* values);
int sap_mm_read_vector(const char* path, int64_t* n, double* values);
const char* sap_mm_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SAP_B200_H */
