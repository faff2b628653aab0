// FP64 kernels of the Krylov loop: SpMV (banded row-major and CSR), BLAS-1
// updates and deterministic fused dot products.
#pragma once

#include "common.cuh"

namespace sapb {

// y = A x for the row-major FP64 band of MVBanded (sap/spmv.h:27-74,
// sap/device/matrix_multiply.cuh:301-350): one warp per row, coalesced
// reads of the row's 2K+1 values.
static __global__ void __launch_bounds__(256)
k_spmv_banded(const double* __restrict__ A, const double* __restrict__ x, double* __restrict__ y, int n, int K) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const long long SW = 2LL * K + 1;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int lo = max(0, i - K), hi = min(n - 1, i + K);
    const double* row = A + (long long)i * SW + K - i;  // row[j] = A(i, j)
    double acc = 0.0;
    for (int j = lo + lane; j <= hi; j += 32) acc += row[j] * x[j];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) y[i] = acc;
  }
}

// y = A x, FP64 CSR by row blocks (the product SpmvCusp delegates to,
// sap/spmv.h:110-121).  The rows are cut on the host into blocks of at most
// kSpmvRows rows and kSpmvNnz entries (csr_row_blocks); a row longer than
// kSpmvNnz is a block of its own.  A CTA streams its block's entries with
// fully coalesced loads of values and column indices, several per thread
// before their gathers of x, keeps the products in shared memory, then one
// thread per row adds its row's products in entry order.  A long row is
// summed by the whole CTA (strided partial sums, then a fixed-order
// reduction).
constexpr int kSpmvRows = 256;   // threads per CTA, rows per block at most
constexpr int kSpmvNnz = 2048;   // entries per block at most (16 KB of products)

static __global__ void __launch_bounds__(kSpmvRows)
k_spmv_csr_blocks(const int* __restrict__ blk, const int* __restrict__ rp, const int* __restrict__ ci,
                  const double* __restrict__ v, const double* __restrict__ x, double* __restrict__ y) {
  __shared__ double prod[kSpmvNnz];
  const int r0 = blk[blockIdx.x], r1 = blk[blockIdx.x + 1];
  const int e0 = rp[r0], cnt = rp[r1] - e0;
  const int t = threadIdx.x;
  if (cnt <= kSpmvNnz) {
    constexpr int U = kSpmvNnz / kSpmvRows;
    int c[U];
    double a[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int k = t + u * kSpmvRows;
      c[u] = k < cnt ? __ldg(ci + e0 + k) : 0;
      a[u] = k < cnt ? __ldg(v + e0 + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int k = t + u * kSpmvRows;
      if (k < cnt) prod[k] = a[u] * __ldg(x + c[u]);
    }
    __syncthreads();
    const int row = r0 + t;
    if (row < r1) {
      const int a0 = rp[row] - e0, a1 = rp[row + 1] - e0;
      double s = 0.0;
      for (int k = a0; k < a1; k++) s += prod[k];
      y[row] = s;
    }
  } else {  // one long row
    double s = 0.0;
    for (int k = t; k < cnt; k += kSpmvRows) s += __ldg(v + e0 + k) * __ldg(x + __ldg(ci + e0 + k));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((t & 31) == 0) prod[t >> 5] = s;
    __syncthreads();
    if (t == 0) {
      double tot = 0.0;
      for (int w = 0; w < kSpmvRows / 32; w++) tot += prod[w];
      y[r0] = tot;
    }
  }
}

// Row blocks of k_spmv_csr_blocks: boundaries b[0] = 0 < b[1] < ... = n, each
// block at most kSpmvRows rows and kSpmvNnz entries, or one longer row.
inline std::vector<int> csr_row_blocks(int n, const int* rp) {
  std::vector<int> b(1, 0);
  int r = 0;
  while (r < n) {
    const int r0 = r;
    while (r < n && r - r0 < kSpmvRows && rp[r + 1] - rp[r0] <= kSpmvNnz) r++;
    if (r == r0) r = r0 + 1;  // a row longer than kSpmvNnz
    b.push_back(r);
  }
  return b;
}

// z = a*x + b*y (cusp::blas::axpby)
static __global__ void k_axpby(int n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                        double* __restrict__ z) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    z[i] = a * x[i] + b * y[i];
}
// y += a*x (cusp::blas::axpy)
static __global__ void k_axpy(int n, double a, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += a * x[i];
}
// z = b - y  (the true-residual recheck, axpby(b, APxx, rr0, 1, -1))
static __global__ void k_sub(int n, const double* __restrict__ b, const double* __restrict__ y, double* __restrict__ z) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = b[i] - y[i];
}

// Up to 4 dot products sum_i x_q[i]*y_q[i] in one pass.  Block partials go to
// `part` (4 * gridDim.x doubles); the last block to finish reduces them in a
// fixed order, so the result is deterministic for a given grid.  `counter`
// must be zero on entry and is zero again on exit.
struct DotArgs {
  const double* x[4];
  const double* y[4];
  int nq;
};

constexpr int kDotBlocks = 296;
constexpr int kDotThreads = 512;
// rows per thread of the size-proportional grid of the standalone dot entry point
constexpr int kDotItems = 16;
inline int dot_grid_for(long long n) {
  long long g = (n + (long long)kDotThreads * kDotItems - 1) / ((long long)kDotThreads * kDotItems);
  return (int)(g < 1 ? 1 : g);
}

static __global__ void __launch_bounds__(kDotThreads)
k_dots(int n, DotArgs a, double* __restrict__ part, unsigned int* __restrict__ counter,
       double* __restrict__ out) {
  __shared__ double red[4][kDotThreads / 32];
  __shared__ bool last;
  double acc[4] = {0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < a.nq) acc[q] += a.x[q][i] * a.y[q][i];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    double v = acc[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (lane == 0) red[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    int q = threadIdx.x;
    double v = 0;
    for (int w = 0; w < kDotThreads / 32; w++) v += red[q][w];
    part[q * gridDim.x + blockIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (last) {
    __threadfence();
    if (threadIdx.x < 4 && threadIdx.x < a.nq) {
      int q = threadIdx.x;
      volatile double* pp = part;
      double v = 0;
      for (int b = 0; b < (int)gridDim.x; b++) v += pp[q * gridDim.x + b];
      out[q] = v;
    }
    if (threadIdx.x == 0) *counter = 0u;
  }
}


// y += a x, then out[0] = y . y, in one pass: the update of the residual
// followed by its norm in BiCGStab(L).  Same grid, thread-to-row mapping and
// reduction order as k_dots, so out[0] equals k_dots(y, y) after k_axpy.
static __global__ void __launch_bounds__(kDotThreads)
k_axpy_sqnorm(int n, double a, const double* __restrict__ x, double* __restrict__ y, double* __restrict__ part,
              unsigned int* __restrict__ counter, double* __restrict__ out) {
  __shared__ double red[kDotThreads / 32];
  __shared__ bool last;
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = y[i] + a * x[i];
    y[i] = v;
    acc += v * v;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) red[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0;
    for (int w = 0; w < kDotThreads / 32; w++) v += red[w];
    part[blockIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (last) {
    __threadfence();
    if (threadIdx.x == 0) {
      volatile double* pp = part;
      double v = 0;
      for (int b = 0; b < (int)gridDim.x; b++) v += pp[b];
      out[0] = v;
      *counter = 0u;
    }
  }
}

// Classical Gram-Schmidt of the Arnoldi step (flexible GMRES), one launch per
// pass instead of one dot and one axpy per basis vector:
//   k_mdot:  h[i] = V_i . w for i < m (blockIdx.y = i); block partials in
//            part[i][blockIdx.x], reduced in block order by the last block of
//            each vector to finish (deterministic for a given grid), whose
//            counter returns to zero;
//   k_maxpy: w[r] -= h[0] V_0[r] + ... in order i = 0..m-1, one row per
//            thread (the basis pointers and h staged in shared memory).
constexpr int kMdotBlocks = 64;
constexpr int kMdotThreads = 256;
constexpr int kMaxBasis = 64;
static __global__ void __launch_bounds__(kMdotThreads)
k_mdot(int n, const double* const* __restrict__ vs, const double* __restrict__ w, double* __restrict__ part,
       unsigned int* __restrict__ ctr, double* __restrict__ h) {
  __shared__ double red[kMdotThreads / 32];
  __shared__ bool last;
  const int i = blockIdx.y;
  const double* v = vs[i];
  double acc = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) acc += v[r] * w[r];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < kMdotThreads / 32; k++) s += red[k];
    part[(size_t)i * gridDim.x + blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(&ctr[i], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    volatile const double* pp = part + (size_t)i * gridDim.x;
    double s = 0.0;
    for (unsigned b = 0; b < gridDim.x; b++) s += pp[b];
    h[i] = s;
    ctr[i] = 0u;
  }
}

static __global__ void k_maxpy(int n, int m, const double* const* __restrict__ vs, const double* __restrict__ h,
                               double* __restrict__ w) {
  __shared__ const double* sv[kMaxBasis];
  __shared__ double sh[kMaxBasis];
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    sv[i] = vs[i];
    sh[i] = h[i];
  }
  __syncthreads();
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double x = w[r];
    for (int i = 0; i < m; i++) x -= sh[i] * sv[i][r];
    w[r] = x;
  }
}

// w <- w / sqrt(nn[0]) when nn[0] > 0 (the Arnoldi normalisation, with the
// norm left on the device)
static __global__ void k_scale_inv_norm(int n, double* __restrict__ w, const double* __restrict__ nn) {
  const double hn = sqrt(nn[0]);
  if (!(hn > 0)) return;
  const double a = 1.0 / hn;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) w[r] = a * w[r] + 0.0 * w[r];
}

// out = a x + b y + c z (cusp::blas::axpbypcz); out may alias an input
static __global__ void k_axpbypcz(int n, double a, const double* x, double b, const double* y, double c,
                                  const double* z, double* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = a * x[i] + b * y[i] + c * z[i];
}

}  // namespace sapb
