// Strided-batched FP32 GEMM on the 5th-generation tensor cores (sm_100a):
//   C_b = alpha A_b B_b + beta C_b,  column-major, b = 0 .. batch-1,
// the products of the wide-band block factorization, spike slabs and
// reduced systems (TF32 inputs, FP32 accumulation in tensor memory).
//
// A persistent grid (at most the CTAs that fit on the SMs at once) walks the
// 128 x BN output tiles of all batch elements; in each CTA
//   warp 0     TMA producer: 128 x 32 tiles of A (four 32 x 32 boxes, M
//              contiguous) and BN x 32 tiles of B (one box, K contiguous)
//              into a ring of shared-memory stages;
//   warp 1     allocates two BN-column accumulators in tensor memory and
//              issues tcgen05.mma (kind::tf32, M = 128, N = BN, K = 8) from
//              one thread; tcgen05.commit frees a stage once its MMAs have
//              read it and hands a finished accumulator to the epilogue;
//   warps 2-5  epilogue: tcgen05.ld of a finished accumulator (warp w reads
//              lanes 32 (w mod 4) ...), alpha / beta, coalesced column
//              stores, then the accumulator is free again: the epilogue of
//              one tile overlaps the MMAs of the next.
// A is read MN-major (M contiguous) and B K-major, which is what column-major
// storage gives without a transpose.  An MN-major TF32 operand must use the
// 128-byte swizzle with 32-byte atoms (TMA SWIZZLE_128B_ATOM_32B, descriptor
// layout SWIZZLE_128B_BASE32B: 4 K-rows of 128 bytes per atom); the K-major
// B uses the 128-byte swizzle with 16-byte atoms (8 rows per atom).  The TMA
// descriptors round FP32 to TF32 (round to nearest) on the way into shared
// memory.  Out-of-range rows and columns of a tile are zero-filled by TMA and
// not stored.
//
// Launches are programmatic dependent launches: a CTA lets the next kernel
// of the stream start its prologue at once, and waits for its predecessor
// (griddepcontrol.wait) before its first global read or write.
//
// Every wait on an mbarrier is bounded: when a wait runs out, the kernel
// raises an error word, drains its own copies and MMAs (again with bounds),
// frees its tensor memory and returns; the host reports the error.
#pragma once

#include <cuda.h>

#include <cstring>
#include <mutex>

#include "common.cuh"

namespace sapb {
namespace umma {

constexpr int kBM = 128;          // tile rows (UMMA M)
constexpr int kBK = 32;           // K per stage: one 128-byte swizzle row of FP32
constexpr int kEpiWarps = 4;
constexpr int kThreads = 32 * (2 + kEpiWarps);
constexpr uint32_t kSpinLimit = 1u << 22;  // polls of one mbarrier wait before giving up

template <int BN>
struct Cfg {
  static_assert(BN == 64 || BN == 128 || BN == 256, "tile width");
  static constexpr int kStages = BN == 256 ? 4 : (BN == 128 ? 3 : 4);
  static constexpr int kABytes = kBM * kBK * 4;  // 16 KB: four 32 x 32 boxes
  static constexpr int kBBytes = BN * kBK * 4;   // BN rows of 128 bytes
  static constexpr int kStage = kABytes + kBBytes;
  static constexpr int kBarBytes = 256;          // full[], empty[], acc_full[2], acc_empty[2], drain, tmem slot, abort
  static constexpr int kSmem = kStages * kStage + kBarBytes + 1024;  // + alignment slack
  static constexpr int kTmemCols = 2 * BN;       // two accumulators; a power of two >= 32
};

// ---- PTX wrappers ---------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// 32 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tc_ld_32cols(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor (tcgen05 "matrix descriptor"): start
// address, leading and stride byte offsets (all >> 4), the sm_100 version
// bit and the layout type (2: 128-byte swizzle with 16-byte atoms, 1: 128-byte
// swizzle with 32-byte atoms).
constexpr uint32_t kLayoutSW128 = 2, kLayoutSW128Base32 = 1;
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  d |= (uint64_t)layout << 61;
  return d;
}
// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, A
// MN-major, B K-major, N = BN, M = 128.
template <int BN>
__device__ __forceinline__ constexpr uint32_t instr_desc() {
  return (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | (0u << 16) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(kBM >> 4) << 24);
}

// Bounded wait; false when the limit ran out or another role aborted.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err) {
  for (uint32_t i = 0; i < kSpinLimit; i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 255u && *abort_flag) return false;
  }
  *abort_flag = 1;
  atomicExch(err, 1);
  return false;
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1)
k_umma_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, float* __restrict__ C,
            int ldc, long long sC, int M, int N, int K, int batch, float alpha, float beta, int* err) {
  using G = Cfg<BN>;
  extern __shared__ unsigned char smem_raw[];
  // stage buffers on a 1024-byte boundary of the shared window (swizzle atoms)
  unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  unsigned char* stage_base = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::kStages * G::kStage);
  constexpr int S = G::kStages;
  // bars: [0, S) full, [S, 2S) empty, [2S, 2S+2) accumulator full,
  // [2S+2, 2S+4) accumulator empty, [2S+4] drain
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int KT = (K + kBK - 1) / kBK;
  const int tiles_m = (M + kBM - 1) / kBM, tiles_n = (N + BN - 1) / BN;
  const int tiles_mn = tiles_m * tiles_n, tiles = tiles_mn * batch;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + S);
  const uint32_t accf0 = smem_u32(bars + 2 * S), acce0 = smem_u32(bars + 2 * S + 2), drain = smem_u32(bars + 2 * S + 4);

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(accf0 + 8 * a, 1);
      mbar_init(acce0 + 8 * a, kEpiWarps);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
  }
  if (warp == 1) {
    __syncwarp();
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)G::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  // the next kernel of the stream may start its prologue
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  if (warp == 0 && lane == 0) {
    // ---- producer ----------------------------------------------------------------
    asm volatile("griddepcontrol.wait;" ::: "memory");  // A and B may come from the previous kernel
    int it = 0;
    for (int t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x) {
      const int bz = t / tiles_mn, r = t - bz * tiles_mn;
      const int m0 = (r % tiles_m) * kBM, n0 = (r / tiles_m) * BN;
      for (int kt = 0; kt < KT; kt++, it++) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        if (!wait_bar(empty0 + 8 * s, ph ^ 1u, abort_flag, err)) break;
        const uint32_t fb = full0 + 8 * s;
        mbar_expect_tx(fb, (uint32_t)G::kStage);
        const uint32_t a_dst = smem_u32(stage_base + (size_t)s * G::kStage);
        const uint32_t b_dst = a_dst + G::kABytes;
        const int k0 = kt * kBK;
#pragma unroll
        for (int i = 0; i < 4; i++) tma_load_3d(a_dst + 4096u * i, &tmA, fb, m0 + 32 * i, k0, bz);
        tma_load_3d(b_dst, &tmB, fb, k0, n0, bz);
      }
    }
    if (*abort_flag) {
      // drain: every stage of the last round still owed bytes by TMA
      for (int j = (it > S ? it - S : 0); j < it; j++) {
        const uint32_t fb = full0 + 8 * (j % S);
        const uint32_t ph = (uint32_t)(j / S) & 1u;
        for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(fb, ph); i++) {
        }
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer --------------------------------------------------------------
    constexpr uint32_t idesc = instr_desc<BN>();
    int it = 0, lt = 0;
    for (int t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x, lt++) {
      const int a = lt & 1;
      const uint32_t aph = (uint32_t)(lt >> 1) & 1u;
      if (!wait_bar(acce0 + 8 * a, aph ^ 1u, abort_flag, err)) break;  // the epilogue has read it
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(a * BN);
      for (int kt = 0; kt < KT; kt++, it++) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        if (!wait_bar(full0 + 8 * s, ph, abort_flag, err)) break;
        tc_fence_after();
        const uint32_t a_base = smem_u32(stage_base + (size_t)s * G::kStage);
        const uint32_t b_base = a_base + G::kABytes;
#pragma unroll
        for (int kk = 0; kk < kBK / 8; kk++) {
          // A: 8 K-rows per instruction = two 512-byte atoms of 4 rows (SBO);
          // the M groups of 32 are the 4096-byte boxes (LBO).  B: 8 K values =
          // 32 bytes along each 128-byte row; 8-row groups 1024 bytes apart.
          const uint64_t ad = smem_desc(a_base + 1024u * kk, 4096u, 512u, kLayoutSW128Base32);
          const uint64_t bd = smem_desc(b_base + 32u * kk, 16u, 1024u, kLayoutSW128);
          tc_mma_tf32(d, ad, bd, idesc, (kt > 0 || kk > 0) ? 1u : 0u);
        }
        tc_commit(empty0 + 8 * s);  // the stage is free once these MMAs have read it
      }
      tc_commit(accf0 + 8 * a);  // the accumulator is complete once all MMAs above are
    }
    // no MMA may still run when the tensor memory is freed
    tc_commit(drain);
    for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(drain, 0u); i++) {
    }
  } else if (warp >= 2) {
    // ---- epilogue ----------------------------------------------------------------
    asm volatile("griddepcontrol.wait;" ::: "memory");  // C may be read or written by the previous kernel
    const int q = warp & 3;  // the TMEM lane quadrant this warp may read
    int lt = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, lt++) {
      const int a = lt & 1;
      const uint32_t aph = (uint32_t)(lt >> 1) & 1u;
      if (!wait_bar(accf0 + 8 * a, aph, abort_flag, err) || *abort_flag) break;
      tc_fence_after();
      const int bz = t / tiles_mn, r = t - bz * tiles_mn;
      const int m0 = (r % tiles_m) * kBM, n0 = (r / tiles_m) * BN;
      const int m = m0 + 32 * q + lane;
      float* Cb = C + (long long)bz * sC;
      for (int c0 = 0; c0 < BN && n0 + c0 < N; c0 += 32) {
        float v[32];
        tc_ld_32cols(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(a * BN + c0), v);
        if (m < M) {
          float* col = Cb + (long long)(n0 + c0) * ldc + m;
          const int nc = min(32, N - n0 - c0);
          // fully unrolled: v stays in registers (predicated by the column count)
          if (beta == 0.f) {
#pragma unroll
            for (int j = 0; j < 32; j++)
              if (j < nc) col[(long long)j * ldc] = alpha * v[j];
          } else {
            // all 32 loads of C first, then the stores: interleaved, every
            // load would wait for the store before it (they may alias)
            float c[32];
#pragma unroll
            for (int j = 0; j < 32; j++) c[j] = j < nc ? col[(long long)j * ldc] : 0.f;
#pragma unroll
            for (int j = 0; j < 32; j++)
              if (j < nc) col[(long long)j * ldc] = alpha * v[j] + beta * c[j];
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce0 + 8 * a);  // this warp is done with the accumulator
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)G::kTmemCols)
                 : "memory");
  }
}

// C = beta C where the product has no K extent (no kernel reads A or B)
static __global__ void k_gemm_scale(float* __restrict__ C, int ldc, long long sC, int M, int N, float beta) {
  float* Cb = C + (long long)blockIdx.z * sC;
  for (int j = blockIdx.y; j < N; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
      float* p = Cb + (long long)j * ldc + i;
      *p = beta == 0.f ? 0.f : beta * *p;
    }
}

// ---- host side -------------------------------------------------------------------
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry-point table (the
// library does not link libcuda)
inline EncodeTiled encode_fn() {
  static EncodeTiled fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<EncodeTiled>(f);
  }();
  return fn;
}

// Whether the tensor-core GEMM can run on this device (sm_100 and the TMA
// descriptor encoder available).
inline bool available() {
  static int avail = -1;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (avail < 0) {
    int dev = 0, major = 0, minor = 0;
    avail = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) == cudaSuccess)
      avail = (major == 10 && minor == 0 && encode_fn() != nullptr) ? 1 : 0;
  }
  return avail == 1;
}

// A 3-D view (rows contiguous, columns at ld, batch at s) as a TMA tensor map
// with box {32, box1, 1}, TF32 rounding, 128-byte swizzle (32-byte atoms for
// an MN-major operand), zero fill.
inline bool make_map(CUtensorMap* map, const float* p, int rows, int cols, int ld, long long s, int batch, int box1,
                     bool mn_major) {
  EncodeTiled enc = encode_fn();
  if (!enc) return false;
  if ((reinterpret_cast<uintptr_t>(p) & 15u) != 0 || ld % 4 != 0 || rows <= 0 || cols <= 0 || batch <= 0) return false;
  long long s_bytes = batch > 1 ? s * 4 : ((long long)ld * cols * 4 + 15) / 16 * 16;
  if (batch > 1 && (s % 4 != 0 || s < (long long)ld * (cols - 1) + rows)) return false;
  if (s_bytes <= 0 || s_bytes >= (1LL << 40) || (long long)ld * 4 >= (1LL << 40)) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)rows, (cuuint64_t)cols, (cuuint64_t)batch};
  const cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)s_bytes};
  const cuuint32_t box[3] = {32u, (cuuint32_t)box1, 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  std::memset(map, 0, sizeof(CUtensorMap));
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32, 3, const_cast<float*>(p), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, mn_major ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN>
inline void set_smem_attr() {
  static bool done = false;  // the first call runs outside any stream capture (see WideBand::init)
  if (!done) {
    SAPB_CUDA(cudaFuncSetAttribute(k_umma_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg<BN>::kSmem));
    done = true;
  }
}

// CTAs of one tile width that fit on the device at once (the persistent grid)
template <int BN>
inline int resident_ctas() {
  static int n = 0;
  if (n == 0) {
    int dev = 0, sms = 0, occ = 0;
    SAPB_CUDA(cudaGetDevice(&dev));
    SAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SAPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_umma_gemm<BN>, kThreads, Cfg<BN>::kSmem));
    n = std::max(1, sms * std::max(1, occ));
  }
  return n;
}

// kernel attributes and grid sizes, set once outside any stream capture
inline void prepare() {
  set_smem_attr<64>();
  set_smem_attr<128>();
  set_smem_attr<256>();
  resident_ctas<64>();
  resident_ctas<128>();
  resident_ctas<256>();
}

template <int BN>
inline void launch_bn(const CUtensorMap& ta, const CUtensorMap& tb, float* C, int ldc, long long sC, int m, int n,
                      int k, float alpha, float beta, int batch, int* err, cudaStream_t st) {
  set_smem_attr<BN>();
  const long long tiles = (long long)((m + kBM - 1) / kBM) * ((n + BN - 1) / BN) * batch;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)std::min<long long>(tiles, resident_ctas<BN>()));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = Cfg<BN>::kSmem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  SAPB_CUDA(cudaLaunchKernelEx(&cfg, k_umma_gemm<BN>, ta, tb, C, ldc, sC, m, n, k, batch, alpha, beta, err));
  SAPB_LAUNCHED();
}

inline int pick_bn(int n) { return n <= 64 ? 64 : (n <= 128 ? 128 : 256); }

// C = alpha A B + beta C for `batch` column-major matrices (A m x k at lda /
// sA, B k x n at ldb / sB, C m x n at ldc / sC).  False (nothing launched)
// when a view does not meet the TMA rules (16-byte aligned base, leading
// dimensions and batch strides multiples of 4 values).
inline bool gemm(int m, int n, int k, float alpha, const float* A, int lda, long long sA, const float* B, int ldb,
                 long long sB, float beta, float* C, int ldc, long long sC, int batch, int* err, cudaStream_t st) {
  if (m <= 0 || n <= 0 || batch <= 0) return true;
  if (k <= 0) {
    if (beta == 1.f) return true;
    k_gemm_scale<<<dim3((m + 255) / 256, std::min(n, 1024), batch), 256, 0, st>>>(C, ldc, sC, m, n, beta);
    SAPB_LAUNCHED();
    return true;
  }
  const int bn = pick_bn(n);
  CUtensorMap ta, tb;
  if (!make_map(&ta, A, m, k, lda, sA, batch, 32, true)) return false;
  if (!make_map(&tb, B, k, n, ldb, sB, batch, bn, false)) return false;
  if (bn == 64) launch_bn<64>(ta, tb, C, ldc, sC, m, n, k, alpha, beta, batch, err, st);
  else if (bn == 128) launch_bn<128>(ta, tb, C, ldc, sC, m, n, k, alpha, beta, batch, err, st);
  else launch_bn<256>(ta, tb, C, ldc, sC, m, n, k, alpha, beta, batch, err, st);
  return true;
}

}  // namespace umma
}  // namespace sapb
