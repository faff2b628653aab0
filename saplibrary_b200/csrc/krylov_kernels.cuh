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

// y = A x, FP64 CSR (the product SpmvCusp delegates to, sap/spmv.h:110-121):
// a group of LANES threads per row.  The row loop runs over warp-uniform
// bases (a warp serves 32 / LANES consecutive rows per step), so every lane
// of a warp takes the same number of steps and the full-mask shuffles never
// name a lane that has left the loop; rows past n contribute nothing.
template <int LANES>
__global__ void __launch_bounds__(256)
k_spmv_csr(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
           const double* __restrict__ x, double* __restrict__ y, int n) {
  constexpr int kRowsPerWarp = 32 / LANES;
  const int lane = threadIdx.x & 31;
  const int sub = lane % LANES;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long stride = (((long long)gridDim.x * blockDim.x) >> 5) * kRowsPerWarp;
  for (long long i0 = warp * kRowsPerWarp; i0 < n; i0 += stride) {
    const long long i = i0 + lane / LANES;
    double acc = 0.0;
    if (i < n)
      for (int p = rp[i] + sub; p < rp[i + 1]; p += LANES) acc += v[p] * __ldg(x + ci[p]);
#pragma unroll
    for (int off = LANES / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, LANES);
    if (sub == 0 && i < n) y[i] = acc;
  }
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


// out = a x + b y + c z (cusp::blas::axpbypcz); out may alias an input
static __global__ void k_axpbypcz(int n, double a, const double* x, double b, const double* y, double c,
                                  const double* z, double* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = a * x[i] + b * y[i] + c * z[i];
}

}  // namespace sapb
