// Checks sapb::div_rcp_fast (a / b from the reciprocal y = 1 / b with
// Markstein's correction, the division of the narrow band factorisation's
// fast path) against the division operator on the GPU, in double and float:
// wherever it reports ok, its quotient must equal a / b bit for bit.
// Operands: uniformly random bit patterns (every exponent, NaN, inf,
// subnormals, zeros), values typical of matrix entries, and exponents near
// the edges of the safe range.  Prints one JSON line with the pair counts,
// the mismatches (must be 0) and how many pairs fell outside the fast
// path's range per class.
#include <cstdio>
#include <cstdlib>

#include "../../saplibrary_b200/csrc/common.cuh"

__device__ unsigned long long mix(unsigned long long x) {  // splitmix64 finaliser
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

template <typename T>
struct Bits;
template <>
struct Bits<double> {
  using U = unsigned long long;
  static constexpr int MANT = 52, BIAS = 1023;
  static __device__ double from(U u) { return __longlong_as_double((long long)u); }
  static __device__ U to(double v) { return (U)__double_as_longlong(v); }
};
template <>
struct Bits<float> {
  using U = unsigned int;
  static constexpr int MANT = 23, BIAS = 127;
  static __device__ float from(U u) { return __uint_as_float(u); }
  static __device__ U to(float v) { return __float_as_uint(v); }
};

// class 0: random bit pattern; 1: uniform in [-10, 10]; 2: exponent within
// `spread` of +-`edge` (unbiased), subnormal or infinite past the range
template <typename T>
__device__ T draw(unsigned long long h, int mode, int edge, int spread) {
  using B = Bits<T>;
  using U = typename B::U;
  if (mode == 0) return B::from((U)h);
  if (mode == 1) return (T)(((double)(h >> 11) * 0x1p-53 - 0.5) * 20.0);
  const int e = ((h >> 60) & 1 ? edge : -edge) + (int)((h >> 40) % (2 * spread + 1)) - spread;
  const int be = e + B::BIAS;
  U mant = (U)(h & ((U(1) << B::MANT) - 1));
  U bits;
  if (be <= 0) bits = mant >> min(-be + 1, B::MANT);
  else if (be >= 2 * B::BIAS + 1) bits = U(2 * B::BIAS + 1) << B::MANT;
  else bits = ((U)be << B::MANT) | mant;
  if ((h >> 63) & 1) bits |= U(1) << (sizeof(U) * 8 - 1);
  return B::from(bits);
}

template <typename T>
__global__ void k_check(int mode_a, int mode_b, int edge, int spread, int per_thread, unsigned long long seed,
                        unsigned long long* counts) {
  using B = Bits<T>;
  const unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  unsigned long long bad = 0, slow = 0;
  for (int i = 0; i < per_thread; i++) {
    const unsigned long long h1 = mix(seed ^ (t * 2654435761ull + i * 0x100000001b3ull));
    const unsigned long long h2 = mix(h1 ^ 0x5851f42d4c957f2dull);
    const T a = draw<T>(h1, mode_a, edge, spread), b = draw<T>(h2, mode_b, edge, spread);
    const T y = T(1) / b;
    bool ok;
    const T q1 = sapb::div_rcp_fast(a, b, y, ok), q2 = a / b;
    if (!ok) slow++;
    else if (B::to(q1) != B::to(q2) && !(q1 != q1 && q2 != q2)) bad++;
  }
  atomicAdd(&counts[0], bad);
  atomicAdd(&counts[1], slow);
}

template <typename T>
void run(int ma, int mb, int edge, int spread, unsigned long long seed, unsigned long long* tot) {
  unsigned long long* c;
  unsigned long long h[2] = {0, 0};
  cudaMalloc(&c, 16);
  cudaMemset(c, 0, 16);
  const int blocks = 148 * 8, threads = 256, per = 16;
  k_check<T><<<blocks, threads>>>(ma, mb, edge, spread, per, seed, c);
  cudaMemcpy(h, c, 16, cudaMemcpyDeviceToHost);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    printf("{\"error\": \"%s\"}\n", cudaGetErrorString(err));
    std::exit(2);
  }
  cudaFree(c);
  tot[0] += (unsigned long long)blocks * threads * per;
  tot[1] += h[0];
  tot[2] += h[1];
  if (ma == 1 && mb == 1) tot[3] += h[1];  // matrix-like values outside the fast path
}

int main() {
  unsigned long long d[4] = {0, 0, 0, 0}, f[4] = {0, 0, 0, 0};
  for (int m = 0; m < 3; m++)
    for (int n = 0; n < 3; n++) {
      run<double>(m, n, 980, 60, 11 + 3 * m + n, d);
      run<double>(m, n, 0, 6, 101 + 3 * m + n, d);
      run<float>(m, n, 110, 30, 211 + 3 * m + n, f);
      run<float>(m, n, 0, 6, 311 + 3 * m + n, f);
    }
  printf("{\"double_pairs\": %llu, \"double_mismatches\": %llu, \"double_outside\": %llu, "
         "\"double_typical_outside\": %llu, \"float_pairs\": %llu, \"float_mismatches\": %llu, "
         "\"float_outside\": %llu, \"float_typical_outside\": %llu}\n",
         d[0], d[1], d[2], d[3], f[0], f[1], f[2], f[3]);
  return (d[1] || f[1]) ? 1 : 0;
}
