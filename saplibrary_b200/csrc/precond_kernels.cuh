// Device kernels of the SPIKE preconditioner (setup and apply).
//
// Storage (kept from the reference because the factor, spike and sweep
// index arithmetic depends on it): each partition's band is column-major
// with 2K+1 entries per column, element (i,j) at (j-start)*(2K+1)+K+(i-j)
// from the partition's base offset (sap/device/data_transfer.cuh:423-495).
// For a constant-bandwidth matrix the partition bases coincide with the
// global layout of the reference.
#pragma once

#include "common.cuh"

namespace sapb {

struct PartDev {
  int start, size, K, ul;  // ul: partition holds UL factors (last one under LU_UL)
  long long boff;          // offset of the partition's first band column
};

struct ChunkDev {
  int part, a, b, pad;     // rows [a, b) of partition `part`
};

struct FactorJob {
  int s, e, K, mirror;     // rows [s, e); mirror = UL factorisation
  int target, pad;         // 0: factors into B, 1: into B2
  long long boff;          // band offset of column s in the target buffer
};

enum { DIR_DOWN = 1, DIR_UP = -1 };

// ---------------------------------------------------------------------------
// Row-major FP64 band (sap/banded_matrix.h layout) -> column-major FP32 band
// (bandedMatrixTranspose, sap/device/data_transfer.cuh:733-770).
template <typename T>
__global__ void k_band_from_rowmajor(const double* __restrict__ A, T* __restrict__ B, int n, int K) {
  const long long SW = 2LL * K + 1;
  const long long total = SW * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long c = e / SW;
    int pos = (int)(e - c * SW);
    long long r = c + pos - K;
    T v = 0.f;
    if (r >= 0 && r < n) v = (T)A[r * SW + (2 * K - pos)];
    B[e] = v;
  }
}

// Diagonal scaling of the TF32 forms: s_r = 2^k with k = -floor(e / 2) for
// |a_rr| = f 2^e (f in [0.5, 1)), so that s_r^2 |a_rr| lies in [0.5, 2)
// (s_r = 1 for a zero or non-finite diagonal).  Powers of two scale without
// rounding, so the factors of S A S are those of A scaled exactly; what
// changes is that the pivot-boost and zero-pivot thresholds see pivots near 1.
template <typename T>
__global__ void k_diag_pow2(const T* __restrict__ B, int n, int K, T* __restrict__ s) {
  const long long SW = 2LL * K + 1;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double d = fabs((double)B[(long long)r * SW + K]);
    int e = 0;
    if (d > 0 && isfinite(d)) frexp(d, &e);
    s[r] = (T)ldexp(1.0, -(e >> 1));
  }
}
// B(i, j) *= s_i s_j over the column-major band
template <typename T>
__global__ void k_band_scale(T* __restrict__ B, int n, int K, const T* __restrict__ s) {
  const long long SW = 2LL * K + 1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < SW * n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long c = e / SW;
    const long long r = c + (e - c * SW) - K;
    if (r >= 0 && r < n) B[e] *= s[r] * s[c];
  }
}

// COO/CSR scatter into the column-major band (copyFromCOOMatrixToBandedMatrix,
// sap/device/data_transfer.cuh:423-448): one thread per row.
template <typename T>
__global__ void k_band_from_csr(const int* __restrict__ rp, const int* __restrict__ ci,
                                const double* __restrict__ v, T* __restrict__ B, int n, int K) {
  const long long SW = 2LL * K + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    for (int p = rp[i]; p < rp[i + 1]; p++) {
      int j = ci[p];
      B[(long long)j * SW + K + (i - j)] = (T)v[p];
    }
  }
}

// Off-diagonal coupling blocks of each interface (copydWV*,
// sap/device/data_transfer.cuh:129-199): B_i[c][r] = A(s-K+c, s+r) for
// r <= c, C_{i+1}[c][r] = A(s+c, s-K+r) for c <= r, both row-major.
template <typename T>
__global__ void k_extract_offdiag(const PartDev* __restrict__ parts, const T* __restrict__ B,
                                  T* __restrict__ offd, int K) {
  const int i = blockIdx.y;
  const int s = parts[i + 1].start;
  const long long SW = 2LL * K + 1;
  const long long KK = (long long)K * K;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < K * K; e += gridDim.x * blockDim.x) {
    int c = e / K, r = e % K;
    T bv = 0.f, cv = 0.f;
    if (r <= c) { long long row = s - K + c, col = s + r; bv = B[col * SW + K + (row - col)]; }
    if (c <= r) { long long row = s + c, col = s - K + r; cv = B[col * SW + K + (row - col)]; }
    offd[(2 * i) * KK + e] = bv;
    offd[(2 * i + 1) * KK + e] = cv;
  }
}

// ---------------------------------------------------------------------------
// Banded LU (or, mirrored, UL) of one partition per CTA, without pivoting,
// with the reference's boosting rule and the row post-divide of the factor
// holding the pivots fused into the write-back
// (bandLU_g32 / blockedBandLU_critical_const_*, bandUL_g32 /
// blockedBandUL_critical_const_*, bandLUUL_post_divide:
// sap/device/factor_band_const.cuh:229-400, 1423-1779).
//
// The active window (columns j..j+K of the pivot j, full 2K+1 band
// positions) lives in shared memory as a ring of W = K+1+D column slots;
// column j+K+D is fetched with cp.async D pivots before it is needed and
// column j-1 is written back (post-divided) while pivot j runs.  Mirrored
// jobs (UL) see the partition with reversed rows and columns, which turns
// the UL elimination into an LU elimination of the mirrored band.
template <typename T, int D>
__global__ void __launch_bounds__(1024)
k_factor_smem(const FactorJob* __restrict__ jobs, T* __restrict__ B, T* __restrict__ B2,
              int do_boost, int* __restrict__ zero_flag, int G) {
  const FactorJob jb = jobs[blockIdx.x];
  const int K = jb.K, SW = 2 * K + 1, np = jb.e - jb.s, W = K + 1 + D;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* sm = reinterpret_cast<T*>(sm_raw);
  T* win = sm;
  T* piv = sm + (size_t)W * SW;
  T* band = (jb.target ? B2 : B) + jb.boff;
  const int tid = threadIdx.x, NT = blockDim.x;
  const bool mir = jb.mirror != 0;
  auto gidx = [&](int i, int p) -> long long {
    int col = mir ? (np - 1 - i) : i;
    int pos = mir ? (2 * K - p) : p;
    return (long long)col * SW + pos;
  };
  for (int i = 0; i < K + D; i++) {
    if (i < np)
      for (int p = tid; p < SW; p += NT) cp_async_val<T>(&win[(i % W) * SW + p], band + gidx(i, p));
    cp_async_commit();
  }
  const int rB = tid % K + 1, gB = tid / K;
  for (int j = 0; j < np; j++) {
    cp_async_wait<D - 1>();
    __syncthreads();
    {
      const int nc = j + K + D;
      const int sl = nc % W;  // == (j-1) % W for j >= 1
      for (int p = tid; p < SW; p += NT) {
        if (j >= 1) {
          T v = win[sl * SW + p];
          if (p < K) {
            int i = j - 1 - K + p;
            if (i >= 0) v /= piv[i % W];
          }
          band[gidx(j - 1, p)] = v;
        }
        if (nc < np) cp_async_val<T>(&win[sl * SW + p], band + gidx(nc, p));
      }
      cp_async_commit();
    }
    const int w = min(K, np - 1 - j);
    const int sj = j % W;
    T p = win[sj * SW + K];
    if (do_boost) p = boost_pivot(p);
    else if (tid == 0 && fabs((double)p) < 1e-7) atomicOr(zero_flag, 1);
    for (int r = tid + 1; r <= w; r += NT) win[sj * SW + K + r] /= p;
    if (tid == 0) piv[sj] = p;
    __syncthreads();
    if (tid == 0) win[sj * SW + K] = p;
    if (gB < G && rB <= w) {
      const T l = win[sj * SW + K + rB];
      int sc = (j + gB + 1) % W;
      for (int c = gB + 1; c <= w; c += G) {
        win[sc * SW + K + rB - c] -= l * win[sc * SW + K - c];
        sc += G;
        if (sc >= W) sc -= W;
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  {
    const int j = np;
    const int sl = (j - 1) % W;
    for (int p = tid; p < SW; p += NT) {
      T v = win[sl * SW + p];
      if (p < K) {
        int i = j - 1 - K + p;
        if (i >= 0) v /= piv[i % W];
      }
      band[gidx(j - 1, p)] = v;
    }
  }
}

// Blocked form of k_factor_smem for K <= 32 R - NB: the same elimination,
// every element receiving the same updates in the same order (hence the same
// factors bit for bit), with two CTA barriers per panel of NB pivots instead
// of two per pivot.
//
// Panel p covers columns j0 = p NB .. j0 + NB - 1.  Warp 0 factors it in
// registers: lane l holds rows j0 + l + 32 t (t < R) of the NB panel columns,
// each pivot is broadcast by a shuffle, its column is divided by it and the
// rest of the panel receives the rank-1 update.  After a barrier the warps
// apply the panel to the K columns right of it, four columns per warp at once
// (the columns' rows in registers, the U element of each pivot broadcast from
// the lane holding that row, each L entry read once from shared memory for
// the four), pivots in order.  While warp 0 factors, the other warps write
// back the previous panel (post-divided by the pivots of its U rows) and
// fetch, with cp.async into the freed slots, the NB columns that panel p + DPF
// will first touch.  The ring holds W = K + NB (1 + DPF) column slots; slots
// advance by additions, with no modulo.
template <typename T, int NB, int R>
__global__ void __launch_bounds__(512)
k_factor_panel(const FactorJob* __restrict__ jobs, T* __restrict__ B, T* __restrict__ B2,
               int do_boost, int* __restrict__ zero_flag, int DPF) {
  constexpr int CPW = 4;  // columns a warp applies a panel to at once
  const FactorJob jb = jobs[blockIdx.x];
  const int K = jb.K, SW = 2 * K + 1, np = jb.e - jb.s, W = K + NB * (1 + DPF);
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* win = reinterpret_cast<T*>(sm_raw);
  T* band = (jb.target ? B2 : B) + jb.boff;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const int ct = tid - 32, nct = blockDim.x - 32;  // copy threads: warps 1..
  const bool mir = jb.mirror != 0;
  auto gidx = [&](int i, int p) -> long long {
    int col = mir ? (np - 1 - i) : i;
    int pos = mir ? (2 * K - p) : p;
    return (long long)col * SW + pos;
  };
  auto wrap = [&](int s) { return s >= W ? s - W : s; };  // for 0 <= s < 2 W
  // column `col` from ring slot `sl` to the band, its U entries post-divided
  // column `col` from ring slot `sl` to the band (its U entries are divided
  // by their rows' pivots afterwards, k_factor_postdiv)
  auto out = [&](int col, int sl, int p) { band[gidx(col, p)] = win[sl * SW + p]; };
  if (ct >= 0) {  // columns [0, K + NB), then one panel's new columns per group; all in slots == column
    for (int g = 0; g < DPF; g++) {
      const int c0 = g == 0 ? 0 : K + g * NB, c1 = min(np, K + (g + 1) * NB);
      for (int e = ct; e < (c1 - c0) * SW; e += nct) {
        const int c = c0 + e / SW, p = e - (c - c0) * SW;
        cp_async_val<T>(&win[c * SW + p], band + gidx(c, p));
      }
      cp_async_commit();
    }
  }
  bool zero_seen = false;
  int j0 = 0, s0 = 0;  // s0 = j0 % W
  for (; j0 < np; j0 += NB, s0 = wrap(s0 + NB)) {
    const int nb = min(NB, np - j0);
    if (DPF == 2) cp_async_wait<1>();
    else cp_async_wait<0>();
    __syncthreads();
    if (warp != 0) {
      // write back panel p-1 and fetch the columns of panel p+DPF into its slots
      // (the thread that reads a slot element issues the copy into it)
      const int nf0 = j0 + DPF * NB + K;
      const int sp = s0 - NB < 0 ? s0 - NB + W : s0 - NB;
      for (int e = ct; e < NB * SW; e += nct) {
        const int c = e / SW, p = e - c * SW, sl = wrap(sp + c);
        if (j0 > 0) out(j0 - NB + c, sl, p);
        if (nf0 + c < np) cp_async_val<T>(&win[sl * SW + p], band + gidx(nf0 + c, p));
      }
      cp_async_commit();
    } else {
      T a[R][NB];
      auto load_panel = [&]() {
#pragma unroll
        for (int c = 0; c < NB; c++) {
          const T* colp = win + wrap(s0 + c) * SW;
#pragma unroll
          for (int t = 0; t < R; t++) {
            const int pos = K + lane + 32 * t - c;  // row j0 + lane + 32 t
            a[t][c] = (c < nb && j0 + lane + 32 * t < np && pos >= 0 && pos <= 2 * K) ? colp[pos] : T(0);
          }
        }
      };
      load_panel();
      // fast path: each quotient from the pivot's reciprocal with Markstein's
      // correction (div_rcp_fast, equal to the division inside its range),
      // without branches; `bad` records a lane whose operands left the range
      bool bad = false;
#pragma unroll
      for (int k = 0; k < NB; k++) {
        if (k < nb) {
          const int w = min(K, np - 1 - (j0 + k));
          T p = __shfl_sync(0xffffffffu, a[0][k], k);
          if (do_boost) p = boost_pivot(p);
          else zero_seen |= fabs((double)p) < 1e-7;
          const T y = T(1) / p;
          T u[NB];
#pragma unroll
          for (int c = k + 1; c < NB; c++) u[c] = __shfl_sync(0xffffffffu, a[0][c], k);
#pragma unroll
          for (int t = 0; t < R; t++) {
            const int rr = lane + 32 * t - k;  // row - pivot row
            const bool in = rr >= 1 && rr <= w;
            bool ok;
            const T l = div_rcp_fast(a[t][k], p, y, ok);
            bad |= in && !ok;
            a[t][k] = rr == 0 ? p : (in ? l : a[t][k]);
#pragma unroll
            for (int c = k + 1; c < NB; c++) {
              if (c - k <= w) {
                const T nv = a[t][c] - l * u[c];
                a[t][c] = in ? nv : a[t][c];
              }
            }
          }
        }
      }
      if (__any_sync(0xffffffffu, bad)) {
        // some quotient left the range: the panel again with the division
        load_panel();
#pragma unroll
        for (int k = 0; k < NB; k++) {
          if (k < nb) {
            const int w = min(K, np - 1 - (j0 + k));
            T p = __shfl_sync(0xffffffffu, a[0][k], k);
            if (do_boost) p = boost_pivot(p);
            T u[NB];
#pragma unroll
            for (int c = k + 1; c < NB; c++) u[c] = __shfl_sync(0xffffffffu, a[0][c], k);
#pragma unroll
            for (int t = 0; t < R; t++) {
              const int rr = lane + 32 * t - k;
              if (rr == 0) {
                a[t][k] = p;
              } else if (rr >= 1 && rr <= w) {
                const T l = a[t][k] / p;
                a[t][k] = l;
#pragma unroll
                for (int c = k + 1; c < NB; c++)
                  if (c - k <= w) a[t][c] -= l * u[c];
              }
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < NB; c++) {
        T* colp = win + wrap(s0 + c) * SW;
#pragma unroll
        for (int t = 0; t < R; t++) {
          const int pos = K + lane + 32 * t - c;
          if (c < nb && j0 + lane + 32 * t < np && pos >= 0 && pos <= 2 * K) colp[pos] = a[t][c];
        }
      }
    }
    __syncthreads();
    // the panel applied to the (up to K) columns right of it, CPW columns per warp at once,
    // pivots in order: x(r, jc) -= L(r, j) U(j, jc)
    const int nt = min(K, np - j0 - nb);
    for (int q0 = warp * CPW; q0 < nt; q0 += nw * CPW) {
      T x[CPW][R];
      T* colp[CPW];
      int kst[CPW];
#pragma unroll
      for (int i = 0; i < CPW; i++) {
        const int q = q0 + i;  // column j0 + nb + q
        colp[i] = win + wrap(s0 + nb + q) * SW;
        kst[i] = q < nt ? max(0, nb + q - K) : NB;
#pragma unroll
        for (int t = 0; t < R; t++) {
          const int pos = K + lane + 32 * t - nb - q;
          x[i][t] = (q < nt && j0 + lane + 32 * t < np && pos >= 0 && pos <= 2 * K) ? colp[i][pos] : T(0);
        }
      }
#pragma unroll
      for (int k = 0; k < NB; k++) {
        if (k < nb) {
          const int w = min(K, np - 1 - (j0 + k));
          const T* lc = win + wrap(s0 + k) * SW + K;
          T L[R];
#pragma unroll
          for (int t = 0; t < R; t++) {
            const int rr = lane + 32 * t - k;
            L[t] = (rr >= 1 && rr <= w) ? lc[rr] : T(0);
          }
#pragma unroll
          for (int i = 0; i < CPW; i++) {
            if (k >= kst[i]) {
              const T U = __shfl_sync(0xffffffffu, x[i][0], k);
#pragma unroll
              for (int t = 0; t < R; t++) {
                const int rr = lane + 32 * t - k;
                if (rr >= 1 && rr <= w) x[i][t] -= L[t] * U;
              }
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < CPW; i++) {
        const int q = q0 + i;
#pragma unroll
        for (int t = 0; t < R; t++) {
          const int pos = K + lane + 32 * t - nb - q;
          if (q < nt && j0 + lane + 32 * t < np && pos >= 0 && pos <= 2 * K) colp[i][pos] = x[i][t];
        }
      }
    }
  }
  if (zero_seen && tid == 0) atomicOr(zero_flag, 1);
  cp_async_wait<0>();
  __syncthreads();
  // the last panel: columns [j0 - NB, np) in slots from s0 - NB on
  const int jl = j0 - NB, sl0 = s0 - NB < 0 ? s0 - NB + W : s0 - NB;
  for (int e = tid; e < (np - jl) * SW; e += blockDim.x) {
    const int c = e / SW;
    out(jl + c, wrap(sl0 + c), e - c * SW);
  }
}

// Post-divide of the panel kernel's factors (bandLUUL_post_divide,
// sap/device/factor_band_const.cuh:1717-1779): every U entry of a job
// (band position p < K of column i with row i - K + p >= 0, in the job's
// own order, mirrored for UL jobs) divided by the pivot of its row, the
// same operands as the one-pivot kernel's write-back.  Pivots (position K)
// are only read.
template <typename T>
__global__ void k_factor_postdiv(const FactorJob* __restrict__ jobs, T* __restrict__ B, T* __restrict__ B2) {
  const FactorJob jb = jobs[blockIdx.y];
  const int K = jb.K, SW = 2 * K + 1, np = jb.e - jb.s;
  T* band = (jb.target ? B2 : B) + jb.boff;
  const bool mir = jb.mirror != 0;
  const long long total = (long long)np * K;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / K), p = (int)(e - (long long)i * K);
    const int r = i - K + p;
    if (r < 0) continue;
    const long long col = mir ? np - 1 - i : i, pos = mir ? 2 * K - p : p, rcol = mir ? np - 1 - r : r;
    band[col * SW + pos] /= band[rcol * SW + K];
  }
}

// Same factorisation operating directly on the band in global memory, for
// half-bandwidths whose window does not fit in shared memory.
template <typename T>
__global__ void __launch_bounds__(1024)
k_factor_global(const FactorJob* __restrict__ jobs, T* __restrict__ B, T* __restrict__ B2,
                int do_boost, int* __restrict__ zero_flag, int G) {
  const FactorJob jb = jobs[blockIdx.x];
  const int K = jb.K, SW = 2 * K + 1, np = jb.e - jb.s;
  T* band = (jb.target ? B2 : B) + jb.boff;
  const int tid = threadIdx.x, NT = blockDim.x;
  const bool mir = jb.mirror != 0;
  auto A = [&](int i, int p) -> T& {
    int col = mir ? (np - 1 - i) : i;
    int pos = mir ? (2 * K - p) : p;
    return band[(long long)col * SW + pos];
  };
  __shared__ T spiv;
  const int rB = tid % K + 1, gB = tid / K;
  for (int j = 0; j < np; j++) {
    __syncthreads();
    if (j >= 1) {  // post-divide the U part of column j-1 (final)
      for (int p = tid; p < K; p += NT) {
        int i = j - 1 - K + p;
        if (i >= 0) A(j - 1, p) /= A(i, K);
      }
    }
    const int w = min(K, np - 1 - j);
    T pv = A(j, K);
    if (do_boost) pv = boost_pivot(pv);
    else if (tid == 0 && fabs((double)pv) < 1e-7) atomicOr(zero_flag, 1);
    for (int r = tid + 1; r <= w; r += NT) A(j, K + r) /= pv;
    if (tid == 0) spiv = pv;
    __syncthreads();
    if (tid == 0) A(j, K) = spiv;
    if (gB < G && rB <= w) {
      const T l = A(j, K + rB);
      for (int c = gB + 1; c <= w; c += G) A(j + c, K + rB - c) -= l * A(j + c, K - c);
    }
  }
  __syncthreads();
  for (int p = tid; p < K; p += NT) {
    int i = np - 1 - K + p;
    if (i >= 0) A(np - 1, p) /= A(i, K);
  }
}

// ---------------------------------------------------------------------------
// Spike tips of the LU_UL method, one CTA per (interface, tip), one thread
// per right-hand-side column (calculateSpikes(B2, WV) and the
// forwardElimLdWV / backwardElimUdWV kernels, sap/precond.h:6232-6287,
// sap/device/sweep_band_const.cuh:585-706), on post-divided factors:
//   V_i = Ut_bb^-1 D_bb^-1 L_bb^-1 B_i   (LU corner of partition i)
//   W_i = Lt_tt^-1 D_tt^-1 U'_tt^-1 C_{i+1}  (UL corner of partition i+1)
template <typename T>
__global__ void k_spikes_luul(const PartDev* __restrict__ parts, int P, const T* __restrict__ B,
                              const T* __restrict__ B2, const T* __restrict__ offd,
                              T* __restrict__ V, T* __restrict__ Wm, int K) {
  const int i = blockIdx.x, which = blockIdx.y, col = threadIdx.x;
  if (col >= K) return;
  const long long SW = 2LL * K + 1, KK = (long long)K * K;
  const int s = parts[i + 1].start;
  auto val = [&](const T* band, long long r, long long c) { return band[c * SW + K + (r - c)]; };
  if (which == 0) {
    T* X = V + i * KK;
    const T* Bm = offd + (2 * i) * KK;
    const long long base = s - K;
    for (int r = 0; r < K; r++) X[r * K + col] = Bm[r * K + col];
    for (int j = 0; j < K - 1; j++) {
      T xj = X[j * K + col];
      for (int t = 1; t < K - j; t++) X[(j + t) * K + col] -= val(B, base + j + t, base + j) * xj;
    }
    for (int j = 0; j < K; j++) X[j * K + col] /= val(B, base + j, base + j);
    for (int j = K - 1; j >= 1; j--) {
      T xj = X[j * K + col];
      for (int t = 1; t <= j; t++) X[(j - t) * K + col] -= val(B, base + j - t, base + j) * xj;
    }
  } else {
    T* X = Wm + i * KK;
    const T* Cm = offd + (2 * i + 1) * KK;
    const T* src = (i + 1 == P - 1) ? B : B2;
    const long long base = s;
    for (int r = 0; r < K; r++) X[r * K + col] = Cm[r * K + col];
    for (int j = K - 1; j >= 1; j--) {
      T xj = X[j * K + col];
      for (int t = 1; t <= j; t++) X[(j - t) * K + col] -= val(src, base + j - t, base + j) * xj;
    }
    for (int j = 0; j < K; j++) X[j * K + col] /= val(src, base + j, base + j);
    for (int j = 0; j < K - 1; j++) {
      T xj = X[j * K + col];
      for (int t = 1; t < K - j; t++) X[(j + t) * K + col] -= val(src, base + j + t, base + j) * xj;
    }
  }
}

// Spike tips of the constant-band LU_only method: V as above; W from full
// sweeps of partition i+1 with K right-hand sides (calculateSpikes_const,
// sap/precond.h:5785-5949), one thread per column, the column kept in a
// global scratch vector of the partition's length.
template <typename T>
__global__ void k_spikes_luonly(const PartDev* __restrict__ parts, const T* __restrict__ B,
                                const T* __restrict__ offd, T* __restrict__ V,
                                T* __restrict__ Wm, T* __restrict__ scratch,
                                long long scratch_stride, int K) {
  const int i = blockIdx.x, which = blockIdx.y, col = threadIdx.x;
  if (col >= K) return;
  const long long SW = 2LL * K + 1, KK = (long long)K * K;
  const int s = parts[i + 1].start;
  auto val = [&](long long r, long long c) { return B[c * SW + K + (r - c)]; };
  if (which == 0) {
    T* X = V + i * KK;
    const T* Bm = offd + (2 * i) * KK;
    const long long base = s - K;
    for (int r = 0; r < K; r++) X[r * K + col] = Bm[r * K + col];
    for (int j = 0; j < K - 1; j++) {
      T xj = X[j * K + col];
      for (int t = 1; t < K - j; t++) X[(j + t) * K + col] -= val(base + j + t, base + j) * xj;
    }
    for (int j = 0; j < K; j++) X[j * K + col] /= val(base + j, base + j);
    for (int j = K - 1; j >= 1; j--) {
      T xj = X[j * K + col];
      for (int t = 1; t <= j; t++) X[(j - t) * K + col] -= val(base + j - t, base + j) * xj;
    }
  } else {
    const int np = parts[i + 1].size;
    T* y = scratch + ((long long)i * K + col) * scratch_stride;
    const T* Cm = offd + (2 * i + 1) * KK;
    for (int r = 0; r < np; r++) y[r] = (r < K) ? Cm[r * K + col] : 0.f;
    for (int j = 0; j < np - 1; j++) {
      T yj = y[j];
      if (yj == 0.f) continue;
      int w = min(K, np - 1 - j);
      for (int t = 1; t <= w; t++) y[j + t] -= val(s + j + t, s + j) * yj;
    }
    for (int j = 0; j < np; j++) y[j] /= val(s + j, s + j);
    for (int j = np - 1; j >= 1; j--) {
      T yj = y[j];
      int w = min(K, j);
      for (int t = 1; t <= w; t++) y[j - t] -= val(s + j - t, s + j) * yj;
    }
    T* X = Wm + i * KK;
    for (int r = 0; r < K; r++) X[r * K + col] = y[r];
  }
}

// Reduced system of each interface: R_i = [[I, V_i], [W_i, I]] has unit
// leading pivots, so its LU reduces to the LU of S_i = I - W_i V_i
// (fullLU_sub_spec + blockedFullLU_phase1..3 + fullLU_post_divide,
// sap/device/factor_band_var.cuh:736-800, 964-1107).  S is row-major, its
// unit-lower L and the post-divided U share the storage, D on the diagonal.
template <typename T>
__global__ void __launch_bounds__(512)
k_reduced_factor(const T* __restrict__ V, const T* __restrict__ Wm, T* __restrict__ S,
                 int K, int do_boost) {
  const int i = blockIdx.x, tid = threadIdx.x, NT = blockDim.x;
  const long long KK = (long long)K * K;
  const T* Vi = V + i * KK;
  const T* Wi = Wm + i * KK;
  T* Si = S + i * KK;
  for (int e = tid; e < K * K; e += NT) {
    int r = e / K, c = e % K;
    T acc = (r == c) ? 1.f : 0.f;
    for (int k = 0; k < K; k++) acc -= Wi[r * K + k] * Vi[k * K + c];
    Si[e] = acc;
  }
  __shared__ T sp;
  for (int j = 0; j < K; j++) {
    __syncthreads();
    T p = Si[j * K + j];
    if (do_boost) p = boost_pivot(p);
    for (int r = j + 1 + tid; r < K; r += NT) Si[r * K + j] /= p;
    if (tid == 0) sp = p;
    __syncthreads();
    if (tid == 0) Si[j * K + j] = sp;
    const int w = K - 1 - j;
    for (int e = tid; e < w * w; e += NT) {
      int r = j + 1 + e / w, c = j + 1 + e % w;
      Si[r * K + c] -= Si[r * K + j] * Si[j * K + c];
    }
  }
  __syncthreads();
  for (int e = tid; e < K * K; e += NT) {
    int r = e / K, c = e % K;
    if (c > r) Si[e] /= Si[r * K + r];
  }
}

// ---------------------------------------------------------------------------
// Chunked partition sweeps.
//
// Every triangular solve of a partition (L or U, unit diagonal) is cut into
// chunks of >= K rows processed in parallel.  The solve of a chunk is an
// affine function of the K "carry" values entering it from the previous
// chunk (in the direction of the solve): tail = T_c * carry + tail0.  A
// setup kernel computes T_c; per apply, pass 1 solves each chunk with a
// zero carry (tail0), a per-partition scan chains the carries, and pass 2/3
// re-solve the chunks with their exact carries.  The result equals the
// serial partition sweep of the reference up to rounding.
//
// Processing-order indexing inside a chunk: xs[0..K) holds the carry rows,
// xs[K..K+m) the chunk rows in the order the solve visits them; the row of
// index u is o + dir*(u-K), with o = a (down) or b-1 (up).  The coefficient
// that propagates row(u) to row(u+t) sits in band column row(u) at position
// K + dir*t.
template <typename T, int PF>
__device__ __forceinline__ void chunk_solve(T* xs, int m, int K, int dir, int o, const T* col0,
                                            int start, int SW, bool carry) {
  const int tid = threadIdx.x, t = tid + 1;
  const int u0 = carry ? 0 : K;
  const int uend = K + m - 1;  // last source index with a target
  T cur[PF], nxt[PF];
  auto ld = [&](int u) -> T {
    int v = u + t;
    if (u < uend && t <= K && v < K + m && v >= K) {
      int row = o + dir * (u - K);
      return __ldg(col0 + (long long)(row - start) * SW + K + dir * t);
    }
    return 0.f;
  };
#pragma unroll
  for (int q = 0; q < PF; q++) cur[q] = ld(u0 + q);
  for (int ub = u0; ub < uend; ub += PF) {
#pragma unroll
    for (int q = 0; q < PF; q++) nxt[q] = ld(ub + PF + q);
#pragma unroll
    for (int q = 0; q < PF; q++) {
      const int u = ub + q;
      __syncthreads();
      if (u < uend) {
        const T xu = xs[u];
        const int v = u + t;
        if (t <= K && v < K + m && v >= K) xs[v] -= cur[q] * xu;
      }
    }
#pragma unroll
    for (int q = 0; q < PF; q++) cur[q] = nxt[q];
  }
  __syncthreads();
}

__device__ __forceinline__ int dir1_of(const PartDev& p) { return p.ul ? DIR_UP : DIR_DOWN; }

// pass 1: first solve of the partition (L for LU partitions, U' for the UL
// partition) with a zero carry; records the chunk's tail.  With vin given,
// the right-hand side is converted from FP64 and stored to F.
template <typename T, int PF>
__global__ void k_pass1(const PartDev* __restrict__ parts, const ChunkDev* __restrict__ chunks,
                        const long long* __restrict__ koff, const T* __restrict__ B,
                        const double* __restrict__ vin, T* __restrict__ F, T* __restrict__ tails,
                        const int* __restrict__ gin, const T* __restrict__ sin) {
  extern __shared__ __align__(16) unsigned char xs_raw[];
  T* xs = reinterpret_cast<T*>(xs_raw);
  const ChunkDev ch = chunks[blockIdx.x];
  const PartDev p = parts[ch.part];
  const int K = p.K, m = ch.b - ch.a, dir = dir1_of(p), o = dir > 0 ? ch.a : ch.b - 1;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    int row = o + dir * i;
    T v;
    if (vin) {
      // leftTrans (precond.h:1535-1544): band row `row` takes input row gin[row], scaled
      if (gin) v = (T)vin[gin[row]] * sin[row];
      else v = sin ? (T)vin[row] * sin[row] : (T)vin[row];
      F[row] = v;
    }
    else v = F[row];
    xs[K + i] = v;
  }
  chunk_solve<T, PF>(xs, m, K, dir, o, B + p.boff, p.start, 2 * K + 1, false);
  for (int i = threadIdx.x; i < K; i += blockDim.x) tails[koff[blockIdx.x] + i] = xs[m + i];
}

// pass 2: first solve with the exact carry, divide by the pivots, store Y,
// then the second solve (opposite direction) of the chunk with a zero carry,
// recording its tail.
template <typename T, int PF>
__global__ void k_pass2(const PartDev* __restrict__ parts, const ChunkDev* __restrict__ chunks,
                        const int* __restrict__ first1, const long long* __restrict__ koff,
                        const T* __restrict__ B, const T* __restrict__ F,
                        const T* __restrict__ carry1, T* __restrict__ Y, T* __restrict__ tails2) {
  extern __shared__ __align__(16) unsigned char xs_raw[];
  T* xs = reinterpret_cast<T*>(xs_raw);
  const int c = blockIdx.x;
  const ChunkDev ch = chunks[c];
  const PartDev p = parts[ch.part];
  const int K = p.K, SW = 2 * K + 1, m = ch.b - ch.a, dir = dir1_of(p), o = dir > 0 ? ch.a : ch.b - 1;
  const bool has_carry = !first1[c];
  const T* col0 = B + p.boff;
  for (int i = threadIdx.x; i < m; i += blockDim.x) xs[K + i] = F[o + dir * i];
  if (has_carry)
    for (int i = threadIdx.x; i < K; i += blockDim.x) xs[i] = carry1[koff[c] + i];
  chunk_solve<T, PF>(xs, m, K, dir, o, col0, p.start, SW, has_carry);
  // divide by the pivots and reverse into the second solve's order
  T* ys = xs + K + m;  // second half of the shared buffer
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    int row = o + dir * i;
    T v = xs[K + i] / col0[(long long)(row - p.start) * SW + K];
    Y[row] = v;
    ys[K + (m - 1 - i)] = v;
  }
  __syncthreads();
  const int dir2 = -dir, o2 = dir2 > 0 ? ch.a : ch.b - 1;
  chunk_solve<T, PF>(ys, m, K, dir2, o2, col0, p.start, SW, false);
  for (int i = threadIdx.x; i < K; i += blockDim.x) tails2[koff[c] + i] = ys[m + i];
}

// pass 3: second solve with the exact carry; writes FP64 (zout) or FP32
// (gout) results in natural row order.
template <typename T, int PF>
__global__ void k_pass3(const PartDev* __restrict__ parts, const ChunkDev* __restrict__ chunks,
                        const int* __restrict__ first2, const long long* __restrict__ koff,
                        const T* __restrict__ B, const T* __restrict__ Y,
                        const T* __restrict__ carry2, double* __restrict__ zout, T* __restrict__ gout,
                        const int* __restrict__ sout, const T* __restrict__ cout) {
  extern __shared__ __align__(16) unsigned char xs_raw[];
  T* xs = reinterpret_cast<T*>(xs_raw);
  const int c = blockIdx.x;
  const ChunkDev ch = chunks[c];
  const PartDev p = parts[ch.part];
  const int K = p.K, SW = 2 * K + 1, m = ch.b - ch.a;
  const int dir2 = -dir1_of(p), o2 = dir2 > 0 ? ch.a : ch.b - 1;
  const bool has_carry = !first2[c];
  for (int i = threadIdx.x; i < m; i += blockDim.x) xs[K + i] = Y[o2 + dir2 * i];
  if (has_carry)
    for (int i = threadIdx.x; i < K; i += blockDim.x) xs[i] = carry2[koff[c] + i];
  chunk_solve<T, PF>(xs, m, K, dir2, o2, B + p.boff, p.start, SW, has_carry);
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    int row = o2 + dir2 * i;
    if (zout) {
      // rightTrans (precond.h:1550-1559): band column `row` is input column sout[row], scaled
      if (sout) zout[sout[row]] = (double)(xs[K + i] * cout[row]);
      else zout[row] = (double)(cout ? xs[K + i] * cout[row] : xs[K + i]);
    } else {
      gout[row] = xs[K + i];
    }
  }
}

// Carry scan of one partition per CTA: carry_{next} = T_c carry_c + tail_c
// along the chunks in the direction of the solve (which = 1: first solve,
// 2: second solve).  T_c is stored column-major (T[k*K + u]).
template <typename T>
__global__ void __launch_bounds__(512)
k_scan(const PartDev* __restrict__ parts, const int* __restrict__ pchunk0, const int* __restrict__ pnchunk,
       const long long* __restrict__ koff, const long long* __restrict__ toff, const T* __restrict__ Tm,
       const T* __restrict__ tails, T* __restrict__ carry, int which, int G) {
  const PartDev p = parts[blockIdx.x];
  const int K = p.K, c0 = pchunk0[blockIdx.x], nc = pnchunk[blockIdx.x];
  if (nc <= 1) return;
  const int dir = (which == 1) ? dir1_of(p) : -dir1_of(p);
  extern __shared__ __align__(16) unsigned char sh_raw[];
  T* sh = reinterpret_cast<T*>(sh_raw);
  T* sig = sh;        // K
  T* red = sh + K;    // G*K
  const int tid = threadIdx.x, u = tid % K, g = tid / K;
  const bool act = g < G;
  for (int step = 0; step < nc - 1; step++) {
    const int c = dir > 0 ? c0 + step : c0 + nc - 1 - step;
    const int cn = dir > 0 ? c + 1 : c - 1;
    T part = 0.f;
    if (act && step > 0) {
      const T* Tc = Tm + toff[c];
      for (int k = g; k < K; k += G) part += Tc[(long long)k * K + u] * sig[k];
    }
    if (act) red[g * K + u] = part;
    __syncthreads();
    if (tid < K) {
      T acc = tails[koff[c] + tid];
      for (int q = 0; q < G; q++) acc += red[q * K + tid];
      carry[koff[cn] + tid] = acc;
      sig[tid] = acc;
    }
    __syncthreads();
  }
}

// Transfer matrices of every chunk for one of the two solves (setup):
// thread k follows a unit carry e_k through the chunk with a zero
// right-hand side and records the chunk's tail, T[k*K + u] = d tail_u / d
// carry_k.  The last K values live in a shared ring of K slots per thread.
template <typename T>
__global__ void k_transfer(const PartDev* __restrict__ parts, const ChunkDev* __restrict__ chunks,
                           const long long* __restrict__ toff, const T* __restrict__ B,
                           T* __restrict__ Tm, int which, T* __restrict__ gring,
                           const int* __restrict__ first) {
  extern __shared__ __align__(16) unsigned char ring_raw[];
  // a chunk that starts its partition in this direction has no carry: its
  // transfer matrix is never read, and its carry rows lie outside the partition
  if (first[blockIdx.x]) return;
  const ChunkDev ch = chunks[blockIdx.x];
  const PartDev p = parts[ch.part];
  const int K = p.K, SW = 2 * K + 1, m = ch.b - ch.a;
  const int NT = blockDim.x;
  // the ring lives in shared memory, or in a per-block global slice when
  // K x blockDim values do not fit
  T* ring = gring ? gring + (long long)blockIdx.x * K * NT : reinterpret_cast<T*>(ring_raw);
  const int dir = (which == 1) ? dir1_of(p) : -dir1_of(p);
  const int o = dir > 0 ? ch.a : ch.b - 1;
  const int k = threadIdx.x;
  if (k < K) {
    for (int u = 0; u < K; u++) ring[u * NT + k] = (u == k) ? T(1) : T(0);
    const T* col0 = B + p.boff;
    for (int v = K; v < K + m; v++) {
      T acc = T(0);
      int slot = (v - 1) % K;
      int row = o + dir * (v - 1 - K);
      for (int t = 1; t <= K; t++) {
        acc -= __ldg(col0 + (long long)(row - p.start) * SW + K + dir * t) * ring[slot * NT + k];
        slot = (slot == 0) ? K - 1 : slot - 1;
        row -= dir;
      }
      ring[(v % K) * NT + k] = acc;
    }
    T* Tc = Tm + toff[blockIdx.x];
    for (int u = 0; u < K; u++) Tc[(long long)k * K + u] = ring[((m + u) % K) * NT + k];
  }
}

// Reduced solve of each interface followed by the purification of the
// interface right-hand sides (partFullFwdSweep/BckSweep + purifyRHS,
// sap/precond.h:5418-5530).  G holds D^-1 f from the first sweep pair;
// F is the FP32 right-hand side the second sweep pair will read.
template <typename T>
__global__ void __launch_bounds__(1024)
k_reduced_apply(const PartDev* __restrict__ parts, const T* __restrict__ V, const T* __restrict__ Wm,
                const T* __restrict__ S, const T* __restrict__ offd, const T* __restrict__ Gv,
                T* __restrict__ F, int K, const int* __restrict__ iface) {
  extern __shared__ __align__(16) unsigned char sh_raw[];
  T* sh = reinterpret_cast<T*>(sh_raw);
  T* xb = sh;
  T* z = sh + K;
  T* x1 = sh + 2 * K;
  const int i = blockIdx.x, r = threadIdx.x;
  const long long KK = (long long)K * K;
  const int s = parts[i + 1].start;
  const T* Vi = V + i * KK;
  const T* Wi = Wm + i * KK;
  const T* Si = S + i * KK;
  const T* Bm = offd + (2 * i) * KK;
  const T* Cm = offd + (2 * i + 1) * KK;
  // band positions of the interface rows: the bottom K rows of partition i
  // and the top K rows of partition i+1 in the first-level order
  const int* map = iface ? iface + (long long)i * 2 * K : nullptr;
  auto pos_b = [&](int q) { return map ? map[q] : s - K + q; };
  auto pos_t = [&](int q) { return map ? map[K + q] : s + q; };
  if (r < K) xb[r] = Gv[pos_b(r)];
  __syncthreads();
  if (r < K) {
    T acc = Gv[pos_t(r)];
    for (int c = 0; c < K; c++) acc -= Wi[r * K + c] * xb[c];
    z[r] = acc;
  }
  for (int j = 0; j < K - 1; j++) {
    __syncthreads();
    T zj = z[j];
    if (r > j && r < K) z[r] -= Si[r * K + j] * zj;
  }
  __syncthreads();
  if (r < K) z[r] /= Si[r * K + r];
  for (int j = K - 1; j >= 1; j--) {
    __syncthreads();
    T zj = z[j];
    if (r < j) z[r] -= Si[r * K + j] * zj;
  }
  __syncthreads();
  if (r < K) {
    T acc = xb[r];
    for (int c = 0; c < K; c++) acc -= Vi[r * K + c] * z[c];
    x1[r] = acc;
  }
  __syncthreads();
  if (r < K) {
    T t1 = 0.f, t2 = 0.f;
    for (int c = 0; c < K; c++) {
      t1 += Bm[r * K + c] * z[c];
      t2 += Cm[r * K + c] * x1[c];
    }
    F[pos_b(r)] -= t1;
    F[pos_t(r)] -= t2;
  }
}

// DB edge weights on the device, as the reference computes them
// (get_csc_matrix + getResidualValues, graph.h:1827-1857, db.cuh:14-37):
// w[e] = log(max_row |a| / |a_e|) in double, one warp per row.
// (as_float: the values are first rounded to FP32, the preconditioner's
// value type, as the host copy the reordering runs on)
__global__ void k_db_weights(const int* __restrict__ rp, const double* __restrict__ a, double* __restrict__ w,
                             double* __restrict__ rowmax, int n, int as_float) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  auto val = [&](int e) { return as_float ? (double)(float)a[e] : a[e]; };
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    double m = 0.0;
    for (int e = rp[i] + lane; e < rp[i + 1]; e += 32) m = fmax(m, fabs(val(e)));
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    for (int e = rp[i] + lane; e < rp[i + 1]; e += 32) w[e] = log(m / fabs(val(e)));
    if (lane == 0) rowmax[i] = m;
  }
}

// Diagonal-block entries (band row j, band column l) into the variable band
// (var::copyFromCOOMatrixToBandedMatrix, data_transfer.cuh:454-495).
template <typename T>
__global__ void k_band_from_coo_var(const int* __restrict__ rows, const int* __restrict__ cols,
                                    const T* __restrict__ vals, long long nz, const PartDev* __restrict__ parts,
                                    const int* __restrict__ part_of_col, T* __restrict__ B) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nz; e += (long long)gridDim.x * blockDim.x) {
    const int j = rows[e], l = cols[e];
    const PartDev p = parts[part_of_col[l]];
    B[p.boff + (long long)(l - p.start) * (2 * p.K + 1) + p.K + (j - l)] = vals[e];
  }
}

// COO entries (band row, column, value) into the constant band (column-major,
// 2K+1 values per column).
template <typename T>
__global__ void k_band_from_coo_const(const int* __restrict__ rows, const int* __restrict__ cols,
                                      const T* __restrict__ vals, long long nz, T* __restrict__ B, int K) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nz; e += (long long)gridDim.x * blockDim.x) {
    const int j = rows[e], l = cols[e];
    B[(long long)l * (2 * K + 1) + K + (j - l)] = vals[e];
  }
}

// update(): out[e] = (T)entries[src[e]] * scale[e] (Precond::update's
// entries x scaleMap, sap/precond.h:760-768).
template <typename T>
__global__ void k_gather_scale(const double* __restrict__ entries, const int* __restrict__ src,
                               const T* __restrict__ scale, long long m, T* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x)
    out[e] = (T)entries[src[e]] * scale[e];
}

// Spike tips of the variable-band method (calculateSpikes_var + spikeSweeps,
// sap/precond.h:5951-6202), computed exactly: V_i = the rows of
// A_i^-1 [0; B_i] at the bottom K first-level rows of partition i, W_i = the
// rows of A_{i+1}^-1 [C_{i+1}; 0] at its top K rows.  The partitions' LU
// factors are in the second-level order, so right-hand sides and tips go
// through the interface position map.  One thread per right-hand-side
// column; the column is swept through the partition in a scratch array
// interleaved by column (coalesced across threads).
template <typename T>
__global__ void k_spikes_var(const PartDev* __restrict__ parts, const T* __restrict__ B,
                             const T* __restrict__ offd, const int* __restrict__ iface, T* __restrict__ V,
                             T* __restrict__ Wm, T* __restrict__ scratch, long long stride, int K) {
  const int i = blockIdx.x, which = blockIdx.y, col = threadIdx.x;
  if (col >= K) return;
  const long long KK = (long long)K * K;
  const PartDev p = parts[i + which];
  const T* M = offd + (2 * i + which) * KK;
  const int* map = iface + (long long)i * 2 * K + (which ? K : 0);
  T* out = (which ? Wm : V) + i * KK;
  bool nz = false;
  for (int r = 0; r < K; r++) nz |= M[r * K + col] != T(0);
  if (!nz) {
    for (int r = 0; r < K; r++) out[r * K + col] = T(0);
    return;
  }
  T* x = scratch + ((long long)(2 * i + which) * stride) * K;  // x[j*K + col], j local to the partition
  const int s = p.start, np = p.size, Kp = p.K, SW = 2 * Kp + 1;
  const T* band = B + p.boff;
  int low = np;
  for (int r = 0; r < K; r++) low = min(low, map[r] - s);
  for (int j = low; j < np; j++) x[(long long)j * K + col] = T(0);
  for (int r = 0; r < K; r++) x[(long long)(map[r] - s) * K + col] = M[r * K + col];
  for (int j = low; j < np - 1; j++) {
    const T xj = x[(long long)j * K + col];
    if (xj == T(0)) continue;
    const int w = min(Kp, np - 1 - j);
    for (int t = 1; t <= w; t++) x[(long long)(j + t) * K + col] -= xj * band[(long long)j * SW + Kp + t];
  }
  for (int j = low; j < np; j++) x[(long long)j * K + col] /= band[(long long)j * SW + Kp];
  for (int j = np - 1; j > low; j--) {
    const T xj = x[(long long)j * K + col];
    const int w = min(Kp, j);
    for (int t = 1; t <= w; t++) x[(long long)(j - t) * K + col] -= xj * band[(long long)j * SW + Kp - t];
  }
  for (int r = 0; r < K; r++) out[r * K + col] = x[(long long)(map[r] - s) * K + col];
}

// K == 0: the band is the diagonal (getSRev, sap/precond.h:1416-1419).
template <typename T>
__global__ void k_diag_apply(const T* __restrict__ B, const double* __restrict__ v, double* __restrict__ z, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    z[i] = (double)((T)v[i] / B[i]);
}

}  // namespace sapb
