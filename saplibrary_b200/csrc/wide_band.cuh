// Wide-band partitions (half-bandwidth of hundreds to thousands): every
// partition is treated as block tridiagonal with bs x bs blocks (bs >= K_p),
//     A_p = tridiag(F_{i-1}, D_i, E_i),
// and factored without pivoting blockwise:
//     D_i <- D_i - L_{i,i-1} U_{i-1,i};  D_i = L_ii U_ii;
//     U_{i,i+1} = L_ii^-1 E_i;  L_{i+1,i} = F_i U_ii^-1.
// These are exactly the L and U factors of the band LU (the LU without
// pivoting is unique), computed as dense block operations: the diagonal block
// LU is recursive and also returns L_ii^-1 and U_ii^-1, so every step except
// the leaves (one CTA each, see k_leaf_lu) is a matrix product.  The apply
// then reduces to batched matrix-vector products per block row:
//     y_i = L_ii^-1 (f_i - L_{i,i-1} y_{i-1}),  x_i = U_ii^-1 (y_i - U_{i,i+1} x_{i+1}).
// Blocks are column-major (element (r, c) at c*bs + r); vectors are padded to
// nb*bs rows per partition, padding rows carry an identity diagonal.
#pragma once

#include <cuda_fp16.h>

#include <cstdlib>
#include <type_traits>

#include "common.cuh"

namespace sapb {

// Granularity (rows) of the block sizes and of the recursion's splits.
constexpr int kLeaf = 32;

// COO entries of the diagonal blocks (row j, col l in band order) into the
// blocks of their partition: D (slot Dm), E = A_{i,i+1} (slot Em), F = A_{i+1,i} (slot Fm).
template <typename T>
__global__ void k_wb_scatter(const int* __restrict__ rows, const int* __restrict__ cols, const T* __restrict__ vals,
                             long long nz, const int* __restrict__ part_of_row, const int* __restrict__ pstart,
                             const int* __restrict__ psize, int bs, int nb, T* __restrict__ Dm, T* __restrict__ Em, T* __restrict__ Fm) {
  const long long BB = (long long)bs * bs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nz;
       e += (long long)gridDim.x * blockDim.x) {
    const int j = rows[e], l = cols[e];
    const int p = part_of_row[j];
    const int a = j - pstart[p], c = l - pstart[p];
    if (c < 0 || c >= psize[p]) continue;  // outside the partition's diagonal block
    const int bi = a / bs, bj = c / bs;
    const long long off = (long long)(c - bj * bs) * bs + (a - bi * bs);
    if (bi == bj) Dm[((long long)p * nb + bi) * BB + off] = vals[e];
    else if (bj == bi + 1) Em[((long long)p * (nb - 1) + bi) * BB + off] = vals[e];
    else if (bj + 1 == bi) Fm[((long long)p * (nb - 1) + bj) * BB + off] = vals[e];
  }
}

// Identity diagonal on the padding rows [psize_p, nb*bs) of every partition.
template <typename T>
__global__ void k_wb_pad(T* __restrict__ Dm, const int* __restrict__ psize, int bs, int nb) {
  const int p = blockIdx.y;
  const long long BB = (long long)bs * bs;
  for (int r = psize[p] + blockIdx.x * blockDim.x + threadIdx.x; r < nb * bs; r += gridDim.x * blockDim.x) {
    const int bi = r / bs, q = r - bi * bs;
    Dm[((long long)p * nb + bi) * BB + (long long)q * bs + q] = T(1);
  }
}

// Band storage (column-major, 2K_p+1 rows per column, element (i, j) of a
// partition at boff + (j-start)*(2K_p+1) + K_p + (i-j)) into the blocks.
template <typename T>
__global__ void k_wb_from_band(const T* __restrict__ B, const long long* __restrict__ boff,
                               const int* __restrict__ kp, const int* __restrict__ psize, int bs, int nb,
                               T* __restrict__ Dm, T* __restrict__ Em, T* __restrict__ Fm) {
  const int p = blockIdx.y;
  const int Kp = kp[p], sz = psize[p];
  const long long SW = 2LL * Kp + 1, BB = (long long)bs * bs;
  const T* Bp = B + boff[p];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)sz * SW;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / SW);
    const int a = c + (int)(e - (long long)c * SW) - Kp;
    if (a < 0 || a >= sz) continue;
    const T v = Bp[e];
    if (v == T(0)) continue;
    const int bi = a / bs, bj = c / bs;
    const long long off = (long long)(c - bj * bs) * bs + (a - bi * bs);
    if (bi == bj) Dm[((long long)p * nb + bi) * BB + off] = v;
    else if (bj == bi + 1) Em[((long long)p * (nb - 1) + bi) * BB + off] = v;
    else if (bj + 1 == bi) Fm[((long long)p * (nb - 1) + bj) * BB + off] = v;
  }
}

// Batched copy of an m x n sub-matrix (column-major, leading dimensions lds/ldd).
template <typename T>
__global__ void k_sub_copy(const T* __restrict__ src, int lds, long long ss, T* __restrict__ dst, int ldd,
                           long long sd, int m, int n, T scale) {
  const int b = blockIdx.z;
  for (int c = blockIdx.y; c < n; c += gridDim.y)
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
      dst[b * sd + (long long)c * ldd + r] = scale * src[b * ss + (long long)c * lds + r];
}

// Batched fill of an m x n sub-matrix with a value.
template <typename T>
__global__ void k_sub_fill(T* __restrict__ dst, int ldd, long long sd, int m, int n, T value) {
  const int b = blockIdx.z;
  for (int c = blockIdx.y; c < n; c += gridDim.y)
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
      dst[b * sd + (long long)c * ldd + r] = value;
}

// Leaf of the recursive block LU: one CTA per batch element factors an n x n
// block (n <= NL) without pivoting (pivots boosted as in the band LU when
// `boost`, else a pivot below 1e-7 raises zero_flag) and writes L^-1 (unit
// lower) to Li and U^-1 (upper) to Ui; M is only read.  Both inverses come
// out of the elimination loop itself (Gauss-Jordan):
//   * eliminating below the pivot in [A | I] turns I into L^-1, stored in
//     place of the multipliers (step j sets G[r][j] = -l_r and updates the
//     columns c < j like the trailing ones);
//   * eliminating below the diagonal of [U^T | I] (row j of U is final at
//     step j) turns I into E with U^-T = diag(U)^-1 E, so U^-1 = E^T diag(U)^-1.
// The working matrix G and E live in registers: thread (ty, tx) of the RY x
// 32 CTA owns rows ty + RY*i and columns tx + 32*k.  Each step the owners of
// pivot row j and pivot column j publish them to shared memory (two buffers,
// so one barrier per step); rows r <= j are skipped per warp.
template <typename T, int NL, int RY>
__global__ void __launch_bounds__(RY * 32) k_leaf_lu(const T* __restrict__ M, int ldm, long long sm,
                                                     T* __restrict__ Li, T* __restrict__ Ui, int ld, long long stride,
                                                     int n, int boost, int* __restrict__ zero_flag) {
  constexpr int TM = NL / RY, TN = NL / 32, NT = RY * 32, SP = NL + 1;
  static_assert(NL % RY == 0 && NL % 32 == 0, "leaf tiling");
  extern __shared__ __align__(16) unsigned char leaf_smem[];
  T* S = reinterpret_cast<T*>(leaf_smem);  // NL x SP staging (row-major)
  T* colj = S + NL * SP;                   // [2][NL] pivot column
  T* rowj = colj + 2 * NL;                 // [2][NL] pivot row of G
  T* erow = rowj + 2 * NL;                 // [2][NL] pivot row of E
  T* piv = erow + 2 * NL;                  // [NL] pivots as used
  const int t = threadIdx.x, tx = t & 31, ty = t >> 5;
  const T* Mb = M + blockIdx.x * sm;
  T* Lb = Li + blockIdx.x * stride;
  T* Ub = Ui + blockIdx.x * stride;
  for (int idx = t; idx < n * n; idx += NT) {
    const int c = idx / n, r = idx - c * n;
    S[r * SP + c] = Mb[(long long)c * ldm + r];
  }
  __syncthreads();
  T g[TM][TN], e[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int k = 0; k < TN; k++) {
      const int r = ty + RY * i, c = tx + 32 * k;
      g[i][k] = (r < n && c < n) ? S[r * SP + c] : (r == c ? T(1) : T(0));
      e[i][k] = r == c ? T(1) : T(0);
    }
  for (int j = 0; j < n; j++) {
    const int b = (j & 1) * NL;
    if (tx == (j & 31)) {  // owners of column j
      const int kj = j >> 5;
#pragma unroll
      for (int i = 0; i < TM; i++) {
        T v = g[i][0];
#pragma unroll
        for (int k = 1; k < TN; k++)
          if (kj == k) v = g[i][k];
        colj[b + ty + RY * i] = v;
      }
    }
    if (ty == j % RY) {  // owners of row j
      const int ij = j / RY;
#pragma unroll
      for (int k = 0; k < TN; k++) {
        T v = g[0][k], w = e[0][k];
#pragma unroll
        for (int i = 1; i < TM; i++)
          if (ij == i) {
            v = g[i][k];
            w = e[i][k];
          }
        rowj[b + tx + 32 * k] = v;
        erow[b + tx + 32 * k] = w;
      }
    }
    __syncthreads();
    T p = rowj[b + j];
    if (boost) p = boost_pivot(p);
    if (t == 0) {
      piv[j] = p;
      if (!boost && fabs((double)p) < 1e-7) atomicOr(zero_flag, 1);
    }
    const T inv = T(1) / p;
    T xr[TN], xe[TN];
#pragma unroll
    for (int k = 0; k < TN; k++) {
      xr[k] = rowj[b + tx + 32 * k];
      xe[k] = erow[b + tx + 32 * k];
    }
#pragma unroll
    for (int i = 0; i < TM; i++) {
      const int r = ty + RY * i;
      if (r > j) {  // uniform across the warp
        const T l = colj[b + r] * inv, m = rowj[b + r] * inv;
#pragma unroll
        for (int k = 0; k < TN; k++) {
          const int c = tx + 32 * k;
          g[i][k] = (c == j) ? -l : g[i][k] - l * xr[k];
          if (c <= j) e[i][k] -= m * xe[k];
        }
      }
    }
  }
  __syncthreads();
  // L^-1: unit diagonal, strict lower part of G
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int k = 0; k < TN; k++) {
      const int r = ty + RY * i, c = tx + 32 * k;
      S[r * SP + c] = r > c ? g[i][k] : (r == c ? T(1) : T(0));
    }
  __syncthreads();
  for (int idx = t; idx < n * n; idx += NT) {
    const int c = idx / n, r = idx - c * n;
    Lb[(long long)c * ld + r] = S[r * SP + c];
  }
  __syncthreads();
  // U^-1 (row c, column r) = E[r][c] / u_rr for c <= r
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int k = 0; k < TN; k++) {
      const int r = ty + RY * i, c = tx + 32 * k;
      S[c * SP + r] = (c <= r && r < n) ? e[i][k] / piv[r] : T(0);
    }
  __syncthreads();
  for (int idx = t; idx < n * n; idx += NT) {
    const int c = idx / n, r = idx - c * n;
    Ub[(long long)c * ld + r] = S[r * SP + c];
  }
}

// CTA rows (warps) and shared memory of k_leaf_lu for a leaf of NL
// (register budget: 2 * TM * TN values per thread).
template <typename T, int NL>
struct LeafShape {
  static constexpr int RY = NL >= 64 ? 16 : 8;
  static constexpr size_t smem = (size_t)(NL * (NL + 1) + 7 * NL) * sizeof(T);
};
// Largest leaf: 32 (measured on the 1M-row workload's 3168 / 3040 blocks:
// TF32 block LU 190 ms with 32, 192 with 64, 215 with 128; FP64 1029 / 1040
// with 32 / 64); SAPB_LEAF = 64 / 128 (128 for FP32 only) overrides.
template <typename T>
inline int leaf_size() {
  const char* e = std::getenv("SAPB_LEAF");
  const int v = e ? std::atoi(e) : 0;
  if (v == 32 || v == 64 || (v == 128 && sizeof(T) == 4)) return v;
  return 32;
}

// Batched dense matrix-vector product with an n x n column-major block:
//   y = A x            (mode 0)
//   y = c - A x        (mode 1)
// one thread per row, x staged in shared memory in tiles.  Batch b uses
// A + b*sA, x + b*sx, c + b*sc, y + b*sy (c may alias y).
template <typename T>
__global__ void __launch_bounds__(256) k_bgemv(const T* A, int ld, long long sA, const T* x, long long sx, const T* c,
                                               long long sc, T* y, long long sy, int n, int mode) {
  __shared__ T xs[256];
  const int b = blockIdx.y;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const T* Ab = A + b * sA;
  const T* xb = x + b * sx;
  T acc = T(0);
  for (int k0 = 0; k0 < n; k0 += 256) {
    const int kk = k0 + threadIdx.x;
    xs[threadIdx.x] = kk < n ? xb[kk] : T(0);
    __syncthreads();
    if (r < n) {
      const int kend = min(256, n - k0);
      const T* col = Ab + (long long)k0 * ld + r;
#pragma unroll 8
      for (int k = 0; k < kend; k++) acc += col[(long long)k * ld] * xs[k];
    }
    __syncthreads();
  }
  if (r < n) y[b * sy + r] = (mode == 1) ? c[b * sc + r] - acc : acc;
}

// Batched matrix-vector product over n x n column-major blocks, for the
// block sweeps and the reduced system:
//   y = A x (mode 0),  y = c - A x (mode 1; c may alias y),
// with tri = 1 (lower: row r reads columns <= r), 2 (upper: columns >= r)
// or 0 (all).  Skipped entries are exact zeros of the factors, so the
// triangular forms read half the bytes.  A CTA of 16 warps owns tiles of
// R = 32*VEC rows; lane l holds rows r0+VEC*l .. r0+VEC*l+VEC-1, so one load
// instruction of a warp is a coalesced column segment of 32*VEC elements
// (16-byte vectors when VEC*sizeof(T) = 16; VEC > 1 needs the leading
// dimension and batch stride to be multiples of VEC and A aligned to
// VEC*sizeof(T)).  The warps split the columns (8 columns in flight per
// warp) and reduce in shared memory in a fixed order.  Tiles are paired j
// with (T-1-j) so triangular work is the same for every CTA.  Batch b uses
// A + b*sA, x + b*sx, c + b*sc, y + b*sy.
// The matrix may be stored as FP16 (MT = __half, 8 rows per 16-byte load)
// with a power-of-two scale per column (see k_blocks_to_half): the kernel
// then reads x_c * cs[b*scs + c] in place of x_c and accumulates in T.
// Chains of these launches are programmatic dependent launches: every CTA
// first lets the next launch of its stream be scheduled
// (griddepcontrol.launch_dependents), then waits for the previous launch to
// complete with its writes visible (griddepcontrol.wait) before it touches
// x, c, y or the column-split scratch; the factor blocks it streams are not
// written by any launch of the apply.
constexpr int kGemvWarps = 16;
template <typename T, int VEC>
struct VecOf;
template <>
struct VecOf<double, 2> { using type = double2; };
template <>
struct VecOf<float, 4> { using type = float4; };
template <>
struct VecOf<__half, 8> { using type = uint4; };
template <typename T>
__device__ __forceinline__ T as_acc(T v) { return v; }
__device__ __forceinline__ float as_acc(__half v) { return __half2float(v); }
template <typename T>
__device__ __forceinline__ void vec_fma(const double2& a, T xv, T* acc) {
  acc[0] += a.x * xv;
  acc[1] += a.y * xv;
}
template <typename T>
__device__ __forceinline__ void vec_fma(const float4& a, T xv, T* acc) {
  acc[0] += a.x * xv;
  acc[1] += a.y * xv;
  acc[2] += a.z * xv;
  acc[3] += a.w * xv;
}
template <typename T>
__device__ __forceinline__ void vec_fma(const uint4& a, T xv, T* acc) {  // 8 x FP16
  const __half2* h = reinterpret_cast<const __half2*>(&a);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const float2 f = __half22float2(h[q]);
    acc[2 * q] += f.x * xv;
    acc[2 * q + 1] += f.y * xv;
  }
}

//
// Column split (gridDim.z = S > 1, for grids with few tiles): CTA s takes
// the s-th contiguous slice of each of its tiles' column ranges and writes
// its R partial sums to ws[((b*ntile + tile)*S + s)*R ..]; the CTA that
// arrives last at the tile's counter (ctr, zero between launches) adds the S
// slices in order s = 0..S-1, writes y and resets the counter.  No CTA waits
// for another.
// One work item of the GEMV: tile pair `pair` (tiles pair and T-1-pair) of
// batch element b, column slice sl of S.  A, x, c, y and cs point at batch
// element b already; b only selects the column-split scratch slots.  CG:
// x and c are read through L2 (written by other CTAs of the same launch).
template <typename T, int VEC, typename MT, bool CG = false>
__device__ __forceinline__ void tgemv_item(int pair, int b, int S, int sl, const MT* Ab, int ld, const T* xb,
                                           const T* cb, T* yb, int n, int mode, int tri, T* ws, unsigned* ctr,
                                           const T* csb, T (*part)[32 * (VEC > 1 ? VEC : 2)],
                                           unsigned& last_cta) {
  constexpr int R = 32 * (VEC > 1 ? VEC : 2);
  const int ntile = (n + R - 1) / R;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // x_c, times the column scale for a scaled FP16 matrix
  auto xs = [&](int col) -> T {
    const T xc = CG ? __ldcg(xb + col) : xb[col];
    if constexpr (std::is_same<MT, T>::value) return xc;
    else return xc * csb[col];
  };
  for (int half = 0; half < 2; half++) {
    const int tile = half == 0 ? pair : ntile - 1 - pair;
    if (half == 1 && tile <= pair) break;
    const int r0 = tile * R;
    int c0 = 0, c1 = n;
    if (tri == 1) c1 = min(n, r0 + R);
    else if (tri == 2) c0 = r0;
    if (S > 1) {
      const int chunk = (c1 - c0 + S - 1) / S;
      const int a = c0 + sl * chunk;
      c1 = min(c1, a + chunk);
      c0 = min(a, c1);
    }
    // 8 independent column loads in flight per warp, then the FMAs
    constexpr int U = 8;
    constexpr int SW = kGemvWarps;  // column stride of a warp
    if constexpr (VEC > 1) {
      using V = typename VecOf<MT, VEC>::type;
      T acc[VEC];
#pragma unroll
      for (int v = 0; v < VEC; v++) acc[v] = T(0);
      const int r = r0 + VEC * lane;
      const int valid = min(VEC, max(0, n - r));
      const MT* base = Ab + r;
      int col = c0 + w;
      if (valid == VEC) {
        for (; col + (U - 1) * SW < c1; col += U * SW) {
          V a[U];
          T xv[U];
#pragma unroll
          for (int u = 0; u < U; u++) {
            a[u] = *reinterpret_cast<const V*>(base + (long long)(col + u * SW) * ld);
            xv[u] = xs(col + u * SW);
          }
#pragma unroll
          for (int u = 0; u < U; u++) vec_fma<T>(a[u], xv[u], acc);
        }
        for (; col < c1; col += SW) vec_fma<T>(*reinterpret_cast<const V*>(base + (long long)col * ld), xs(col), acc);
      } else {
        for (; col < c1; col += SW) {
          const T xv = xs(col);
          for (int v = 0; v < valid; v++) acc[v] += as_acc(base[(long long)col * ld + v]) * xv;
        }
      }
#pragma unroll
      for (int v = 0; v < VEC; v++) part[w][VEC * lane + v] = acc[v];
    } else {
      T acc0 = T(0), acc1 = T(0);
      const int ra = r0 + lane, rb = r0 + 32 + lane;
      const bool va = ra < n, vb = rb < n;
      const MT* pa = Ab + (va ? ra : 0);
      const MT* pb = Ab + (vb ? rb : 0);
      int col = c0 + w;
      for (; col + (U - 1) * SW < c1; col += U * SW) {
        T a0[U], a1[U], xv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const long long o = (long long)(col + u * SW) * ld;
          a0[u] = va ? as_acc(pa[o]) : T(0);
          a1[u] = vb ? as_acc(pb[o]) : T(0);
          xv[u] = xs(col + u * SW);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
          acc0 += a0[u] * xv[u];
          acc1 += a1[u] * xv[u];
        }
      }
      for (; col < c1; col += SW) {
        const T xv = xs(col);
        const long long o = (long long)col * ld;
        if (va) acc0 += as_acc(pa[o]) * xv;
        if (vb) acc1 += as_acc(pb[o]) * xv;
      }
      part[w][lane] = acc0;
      part[w][32 + lane] = acc1;
    }
    __syncthreads();
    if (S == 1) {
      for (int q = threadIdx.x; q < R; q += blockDim.x) {
        const int r = r0 + q;
        T s = T(0);
#pragma unroll
        for (int k = 0; k < kGemvWarps; k++) s += part[k][q];
        if (r < n) yb[r] = (mode == 1) ? (CG ? __ldcg(cb + r) : cb[r]) - s : s;
      }
    } else {
      const long long slot = (long long)b * ntile + tile;
      for (int q = threadIdx.x; q < R; q += blockDim.x) {
        T s = T(0);
#pragma unroll
        for (int k = 0; k < kGemvWarps; k++) s += part[k][q];
        ws[(slot * S + sl) * R + q] = s;
      }
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) last_cta = (atomicAdd(&ctr[slot], 1u) == (unsigned)(S - 1));
      __syncthreads();
      if (last_cta) {
        __threadfence();
        for (int q = threadIdx.x; q < R; q += blockDim.x) {
          const int r = r0 + q;
          T s = T(0);
          for (int k = 0; k < S; k++) s += __ldcg(ws + (slot * S + k) * R + q);
          if (r < n) yb[r] = (mode == 1) ? (CG ? __ldcg(cb + r) : cb[r]) - s : s;
        }
        if (threadIdx.x == 0) ctr[slot] = 0u;
      }
    }
    __syncthreads();
  }
}

// (three CTAs per SM for the vector forms: 16 warps each, <= 42 registers)
template <typename T, int VEC, typename MT = T>
__global__ void __launch_bounds__(kGemvWarps * 32, VEC > 1 ? 3 : 1) k_tgemv(const MT* A, int ld, long long sA, const T* x, long long sx,
                                                           const T* c, long long sc, T* y, long long sy, int n,
                                                           int mode, int tri, T* ws, unsigned* ctr,
                                                           const T* cs = nullptr, long long scs = 0) {
  constexpr int R = 32 * (VEC > 1 ? VEC : 2);
  __shared__ T part[kGemvWarps][R];
  __shared__ unsigned last_cta;
  const int b = blockIdx.y;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  tgemv_item<T, VEC, MT>((int)blockIdx.x, b, (int)gridDim.z, (int)blockIdx.z, A + b * sA, ld, x + b * sx,
                         c ? c + b * sc : nullptr, y + b * sy, n, mode, tri, ws, ctr, cs ? cs + b * scs : nullptr,
                         part, last_cta);
}

// Barrier of the `n` CTAs of one group (a counter and a generation word in
// global memory, zero before the first use).  The wait is bounded: after
// kBarrierSpins polls it raises *err and returns false.
constexpr long long kBarrierSpins = 1LL << 22;
__device__ __forceinline__ bool group_barrier(unsigned* cnt, unsigned* gen, unsigned n, int* err) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    const unsigned g = *reinterpret_cast<volatile unsigned*>(gen);
    __threadfence();
    if (atomicAdd(cnt, 1u) == n - 1) {
      *cnt = 0u;
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      long long it = 0;
      while (*reinterpret_cast<volatile unsigned*>(gen) == g) {
        if (++it > kBarrierSpins || *reinterpret_cast<volatile int*>(err)) {
          atomicOr(err, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  return __syncthreads_and(ok) != 0;
}

// One whole block sweep (x <- A_p^-1 x for every partition) as a single
// cooperative launch: partition p is served by the G CTAs of group p, which
// run its 4 nb - 2 block-row GEMVs (the steps of solve_blocks_part) with a
// group barrier between steps, S column slices per tile pair (items =
// pairs * S per step, spread over the group).  Partitions do not wait for
// each other.  Factor blocks: L_ii^-1 at Li + (p nb + i) BB, L_{i+1,i} at
// Lo + (p (nb-1) + i) BB, likewise U; their column scales (FP16 copies) at
// cs* + (block index) bs.  bar holds 2 words per partition; err is raised by
// a barrier that timed out (the kernel then returns).  stall > 0 makes every
// group barrier wait for that many CTAs more than the group has, so that the
// bounded wait runs out (tests of the timeout path only).
template <typename T, int VEC, typename MT>
__global__ void __launch_bounds__(kGemvWarps * 32, 3) k_sweep(const MT* __restrict__ Li, const MT* __restrict__ Ui,
                                                              const MT* __restrict__ Lo, const MT* __restrict__ Uo,
                                                              const T* csL, const T* csU, const T* csLo, const T* csUo,
                                                              T* x, T* y, T* t, int nb, int bs, long long BB,
                                                              long long plen, int G, int S, T* ws, unsigned* ctr,
                                                              unsigned* bar, int* err, int stall) {
  constexpr int R = 32 * (VEC > 1 ? VEC : 2);
  __shared__ T part[kGemvWarps][R];
  __shared__ unsigned last_cta;
  const int p = blockIdx.x / G, g = blockIdx.x - p * G;
  const int ntile = (bs + R - 1) / R, pairs = (ntile + 1) / 2, items = pairs * S;
  T* xp = x + p * plen;
  T* yp = y + p * plen;
  T* tp = t + p * plen;
  const long long bd = (long long)p * nb, bo = (long long)p * (nb - 1);
  const bool scaled = !std::is_same<MT, T>::value;
  const int steps = 4 * nb - 2;
  for (int s = 0; s < steps; s++) {
    const MT* A;
    const T *xv, *cv = nullptr, *cs = nullptr;
    T* yv;
    int mode = 0, tri;
    if (s < 2 * nb - 1) {  // forward: y_i = L_ii^-1 (x_i - L_{i,i-1} y_{i-1})
      const int i = (s + 1) / 2;
      if (s & 1) {
        A = Lo + (bo + i - 1) * BB;
        cs = scaled ? csLo + (bo + i - 1) * bs : nullptr;
        xv = yp + (long long)(i - 1) * bs;
        cv = xp + (long long)i * bs;
        yv = tp;
        mode = 1;
        tri = 2;
      } else {
        A = Li + (bd + i) * BB;
        cs = scaled ? csL + (bd + i) * bs : nullptr;
        xv = i > 0 ? tp : xp;
        yv = yp + (long long)i * bs;
        tri = 1;
      }
    } else {  // backward: x_i = U_ii^-1 (y_i - U_{i,i+1} x_{i+1})
      const int s2 = s - (2 * nb - 1), k = (s2 + 1) / 2, i = nb - 1 - k;
      if (s2 & 1) {
        A = Uo + (bo + i) * BB;
        cs = scaled ? csUo + (bo + i) * bs : nullptr;
        xv = xp + (long long)(i + 1) * bs;
        cv = yp + (long long)i * bs;
        yv = tp;
        mode = 1;
        tri = 1;
      } else {
        A = Ui + (bd + i) * BB;
        cs = scaled ? csU + (bd + i) * bs : nullptr;
        xv = k > 0 ? tp : yp + (long long)i * bs;
        yv = xp + (long long)i * bs;
        tri = 2;
      }
    }
    for (int it = g; it < items; it += G)
      tgemv_item<T, VEC, MT, true>(it / S, p, S, it % S, A, bs, xv, cv, yv, bs, mode, tri, ws, ctr, cs, part,
                                   last_cta);
    if (!group_barrier(bar + 2 * p, bar + 2 * p + 1, (unsigned)(G + stall), err)) return;
  }
}

// rows per tile of k_tgemv<T, VEC>
template <typename T, int VEC>
constexpr int tgemv_rows() { return 32 * (VEC > 1 ? VEC : 2); }

// FP16 copies of n x n column-major blocks (block b at A + b*BB) for the
// apply, as block floating point: column c is stored as A[:, c] * 2^k_c with
// its largest magnitude in [2^14, 2^15) and cs[b*n + c] = 2^-k_c (a zero
// column gets scale 1).  Only the rows k_tgemv reads for the block's
// triangle are written: tri 1 (lower) rows from the start of the R-row tile
// holding row c, tri 2 (upper) rows up to the end of that tile.  One warp
// per column.
template <typename T, int R>
__global__ void k_blocks_to_half(const T* __restrict__ A, __half* __restrict__ H, T* __restrict__ cs, int n,
                                 long long BB, int tri) {
  const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= n) return;
  const long long o = (long long)blockIdx.y * BB + (long long)c * n;
  const int t0 = (c / R) * R;
  const int r0 = tri == 1 ? t0 : 0, r1 = tri == 2 ? min(n, t0 + R) : n;
  float m = 0.f;
  for (int r = r0 + lane; r < r1; r += 32) m = fmaxf(m, fabsf((float)A[o + r]));
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, d));
  int e = 0;
  if (m > 0.f) {
    frexpf(m, &e);  // m = f * 2^e, f in [0.5, 1)
    e = max(e, -100);
  }
  const float up = m > 0.f ? ldexpf(1.f, 15 - e) : 1.f;
  for (int r = r0 + lane; r < r1; r += 32) H[o + r] = __float2half_rn((float)A[o + r] * up);
  if (lane == 0) cs[(long long)blockIdx.y * n + c] = m > 0.f ? (T)ldexpf(1.f, e - 15) : T(1);
}

// Nonzero columns of the coupling blocks: flag[blk][c] = any row of column c
// of row-major K x K block blk (blk = 2t + which) is nonzero.
template <typename T>
__global__ void k_nz_cols(const T* __restrict__ offd, int K, int* __restrict__ flag) {
  const int blk = blockIdx.y;
  const long long KK = (long long)K * K;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < K; c += gridDim.x * blockDim.x) {
    const T* M = offd + blk * KK + c;
    int nz = 0;
    for (int r = 0; r < K && !nz; r++) nz = M[(long long)r * K] != T(0);
    flag[(long long)blk * K + c] = nz;
  }
}

// Right-hand sides of the spike solves: column jj of interface t's slab is
// coupling-block column cols[t][j0+jj], placed at the interface rows
// pos[t][k] of the partition's block vector (X pre-zeroed).
template <typename T>
__global__ void k_spike_rhs(const T* __restrict__ offd, int which, int K, const int* __restrict__ cols, int ncol,
                            int j0, const int* __restrict__ pos, T* __restrict__ X, long long sX, long long plen) {
  const int jj = blockIdx.x, t = blockIdx.y;
  const int col = (j0 + jj < ncol) ? cols[(long long)t * ncol + j0 + jj] : -1;
  if (col < 0) return;
  const long long KK = (long long)K * K;
  const T* M = offd + (2LL * t + which) * KK + col;
  for (int k = threadIdx.x; k < K; k += blockDim.x)
    X[t * sX + jj * plen + pos[(long long)t * K + k]] = M[(long long)k * K];
}

// Spike tips out of the solved slab: element (k, col) of out[t], column-major
// with leading dimension ldo and batch stride so.
template <typename T>
__global__ void k_spike_tips(const T* __restrict__ X, long long sX, long long plen, const int* __restrict__ cols,
                             int ncol, int j0, const int* __restrict__ pos, int K, int ldo, long long so,
                             T* __restrict__ out) {
  const int jj = blockIdx.x, t = blockIdx.y;
  const int col = (j0 + jj < ncol) ? cols[(long long)t * ncol + j0 + jj] : -1;
  if (col < 0) return;
  for (int k = threadIdx.x; k < K; k += blockDim.x)
    out[t * so + (long long)col * ldo + k] = X[t * sX + jj * plen + pos[(long long)t * K + k]];
}

// Row-major coupling block (2t + which) -> column-major out[t] (leading
// dimension ldo, batch stride so), via 32x32 tiles.
template <typename T>
__global__ void k_couple_colmajor(const T* __restrict__ offd, int which, int K, int ldo, long long so,
                                  T* __restrict__ out) {
  __shared__ T tile[32][33];
  const int t = blockIdx.z;
  const long long KK = (long long)K * K;
  const T* M = offd + (2LL * t + which) * KK;
  T* O = out + t * so;
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < K && c < K) ? M[(long long)r * K + c] : T(0);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (r < K && c < K) O[(long long)c * ldo + r] = tile[threadIdx.x][i];
  }
}

// Band-order vector <-> padded block vectors of the partitions.
template <typename T>
__global__ void k_wb_to_blocks(const T* __restrict__ v, T* __restrict__ out, const int* __restrict__ pstart,
                               const int* __restrict__ psize, long long plen) {
  const int p = blockIdx.y;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < plen; r += (long long)gridDim.x * blockDim.x)
    out[p * plen + r] = r < psize[p] ? v[pstart[p] + r] : T(0);
}
template <typename T>
__global__ void k_wb_from_blocks(const T* __restrict__ in, T* __restrict__ v, const int* __restrict__ pstart,
                                 const int* __restrict__ psize, long long plen) {
  const int p = blockIdx.y;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < psize[p];
       r += (long long)gridDim.x * blockDim.x)
    v[pstart[p] + r] = in[p * plen + r];
}


// dst[idx[e]] = vals[e]  /  dst[e] = src[idx[e]]   (64-bit indices; idx < 0 gives 0)
template <typename T>
__global__ void k_scatter_idx(const long long* __restrict__ idx, const T* __restrict__ vals, long long m,
                              T* __restrict__ dst) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x)
    dst[idx[e]] = vals[e];
}
template <typename T>
__global__ void k_gather_idx(const T* __restrict__ src, const long long* __restrict__ idx, long long m,
                             T* __restrict__ dst) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x)
    dst[e] = idx[e] >= 0 ? src[idx[e]] : T(0);
}

// leftTrans into the band-order right-hand side: F[row] = T(v[gin[row]]) * sin[row]
template <typename T>
__global__ void k_wb_in(const double* __restrict__ v, const int* __restrict__ gin, const T* __restrict__ sin,
                        T* __restrict__ F, int n) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    F[r] = gin ? (T)v[gin[r]] * sin[r] : (sin ? (T)v[r] * sin[r] : (T)v[r]);
}
// rightTrans out of the padded block vectors: z[sout[row]] = x(row) * cout[row]
template <typename T>
__global__ void k_wb_out(const T* __restrict__ xb, const int* __restrict__ rowpart, const int* __restrict__ pstart,
                         long long plen, const int* __restrict__ sout, const T* __restrict__ cout,
                         double* __restrict__ z, int n) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int p = rowpart[r];
    const T x = xb[p * plen + (r - pstart[p])];
    if (sout) z[sout[r]] = (double)(x * cout[r]);
    else z[r] = (double)(cout ? x * cout[r] : x);
  }
}

// dst[didx[e]] = src[sidx[e]]
template <typename T>
__global__ void k_move_idx(const T* __restrict__ src, const long long* __restrict__ sidx,
                           const long long* __restrict__ didx, long long m, T* __restrict__ dst) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x)
    dst[didx[e]] = src[sidx[e]];
}

// S = I (K x K column-major with leading dimension ld, per batch element;
// padding rows zero)
template <typename T>
__global__ void k_identity(T* __restrict__ S, int K, int ld, long long stride) {
  const int b = blockIdx.y;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)ld * K;
       e += (long long)gridDim.x * blockDim.x)
    S[b * stride + e] = (e % ld == e / ld) ? T(1) : T(0);
}

}  // namespace sapb
